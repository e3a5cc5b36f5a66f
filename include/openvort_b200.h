/*
 * openvort_b200.h - C ABI of libov_gpu.so, the B200 (sm_100a) implementation
 * of OpenVort's Schwarz vortex-filament velocity and RK4 path.
 *
 * Part 1 keeps the reference's own data layouts and prototypes so the library
 * is a drop-in for the reference's hot path: a program built from the
 * reference's remaining C files (main.c, reconnection, remeshing, I/O) links
 * against libov_gpu.so instead of tangle.c's velocity functions, octree.c and
 * vortex_dynamics.c's stepping.  Every declaration cites the reference
 * interface it replaces (paths relative to the OpenVort checkout).
 *
 * Part 2 adds entry points the reference has no counterpart for: device
 * selection and error reporting, precision control, a device-resident state
 * for multi-step runs, batched independent systems, point queries, and the
 * adjoint.
 *
 * Error convention: the reference's functions return void and abort through
 * error() (src/util.c:29-34).  Here every failure (no GPU, CUDA error, bad
 * input, non-finite result, tree too deep, spin-wait limit) is recorded in a
 * per-thread status read by ov_last_error(), printed to stderr, and, when the
 * environment variable OV_ABORT_ON_ERROR=1, aborts like the reference.
 * Outputs of a failed call are not written.  There is no CPU fallback.
 */
#ifndef OPENVORT_B200_H
#define OPENVORT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ===================================================================== */
/* Part 1: reference-compatible layouts and prototypes                    */
/* ===================================================================== */

/* The include guards below are the reference headers' own, so this header
 * and the reference's headers can be included in either order. */
#ifndef VEC3_MATHS_H
#define VEC3_MATHS_H
/* include/vec3_maths.h:23-68 */
struct vec3d { double p[3]; };
struct mat3d { double m[3][3]; };
struct segment { struct vec3d r1, r2; };
typedef enum _wt { WALL_OPEN, WALL_PERIODIC, WALL_MIRROR } wall_type;
typedef enum _fc { NOT_A_FACE = -1, X_L, X_H, Y_L, Y_H, Z_L, Z_H } boundary_faces;
struct domain_box {
  struct vec3d bottom_left_back;
  struct vec3d top_right_front;
  wall_type wall[6];
};
#endif

#ifndef TANGLE_H
#define TANGLE_H
/* include/tangle.h:28-106 */
typedef enum _ns_e { EMPTY = -1, FREE, PINNED, PINNED_SLIP } node_status_t;
typedef struct _ns { node_status_t status; boundary_faces pin_wall; } node_status;
struct neighbour_t { int forward; int reverse; };
struct image_tangle { int shift[3]; int reflect; };
struct boundary_images { const struct image_tangle *images; int n; };
struct tangle_state {
  struct vec3d *vnodes;
  struct vec3d *vnodes_new;
  struct vec3d *vels;
  struct vec3d *vs;
  struct vec3d *tangents;
  struct vec3d *normals;
  double *dxi;
  int *recalculate;
  struct neighbour_t *connections;
  node_status *status;
  struct domain_box box;
  struct boundary_images bimg;
  int N;
  int next_free;
  int total_free;
};

/* boundary image tables (include/tangle.h:62-77, src/boundary_images.c).
 * Same images, order and counts as the reference, except wall_1_6: the
 * reference declares n=6 over a 5-entry array (reads past its end); here
 * n=5. */
extern const struct boundary_images open_boundaries;
extern const struct boundary_images periodic_6;
extern const struct boundary_images periodic_18;
extern const struct boundary_images periodic_26;
extern const struct boundary_images periodic_z_open_xy;
extern const struct boundary_images wall_1_open;
extern const struct boundary_images wall_1_6;
extern const struct boundary_images wall_1_18;
extern const struct boundary_images wall_1_26;
extern const struct boundary_images wall_2_4;
extern const struct boundary_images wall_2_2;
extern const struct boundary_images wall_2_26;
extern const struct boundary_images channel_z;

struct octree;

/* image point of r (include/tangle.h:116-117, src/tangle.c:39-79) */
struct vec3d shifted(const struct image_tangle *shift,
                     const struct tangle_state *tangle, const struct vec3d *r);
/* include/tangle.h:119-120, src/tangle.c:245-480,704-727.
 * update_tangents_normals computes dxi, tangents and normals of every node on
 * the GPU.  update_tangent_normal(k) computes the same for the whole tangle
 * from the current positions and writes back node k's tangent and normal. */
void update_tangent_normal(struct tangle_state *tangle, size_t k);
void update_tangents_normals(struct tangle_state *tangle);
/* include/tangle.h:128, src/tangle.c:686-702: velocities of all nodes
 * (LIA + external + direct or Barnes-Hut Biot-Savart + boundary images +
 * hyperfriction + mutual friction).  tree: NULL builds a tree internally when
 * global_use_BH; otherwise a tree from octree_build. */
void update_velocities(struct tangle_state *tangle, double t, struct octree *tree);
/* include/tangle.h:136, src/tangle.c:583-684: one node (used by the
 * reference's reconnection).  One GPU launch per call. */
void update_velocity(struct tangle_state *tangle, int k, double t, struct octree *tree);
/* include/tangle.h:142,152-153, src/tangle.c:553-581 */
struct vec3d calculate_vs(struct tangle_state *tangle, struct vec3d r, int skip);
struct vec3d calculate_vs_shift(const struct tangle_state *tangle, struct vec3d r,
                                int skip, const struct vec3d *shift,
                                const int *use_only_points, const int Npoints);
#endif /* TANGLE_H */

#ifndef INCLUDE_OCTREE_H_
#define INCLUDE_OCTREE_H_
/* include/octree.h:36-48.  struct octree is opaque here: the tree lives in
 * device memory.  Only the reference's octree.c reads its fields, and this
 * library replaces octree.c.  The tree keeps a snapshot of the node
 * positions taken by octree_build. */
struct octree *octree_build(const struct tangle_state *tangle, int quadtree);
void octree_destroy(struct octree *tree);
void octree_get_vs(const struct octree *tree, const struct vec3d *r,
                   double resolution, struct vec3d *res, int skip);
#endif

#ifndef VORTEX_DYNAMICS
#define VORTEX_DYNAMICS
/* include/vortex_dynamics.h:47-49, src/vortex_dynamics.c:36-121.
 * rk4_step needs tangle->vels to hold the velocities at the current
 * positions (as the reference does) and updates tangle->vnodes only. */
void euler_step(struct tangle_state *tangle, double dt);
void rk4_step(struct tangle_state *tangle, double t, double dt);
#endif

#ifndef EXTERNAL_VELOCITY_H
#define EXTERNAL_VELOCITY_H
/* include/external_velocity.h:54-90.  The library reads vn_conf / vs_conf /
 * vb_conf by their name and parameters (the host function pointer cannot run
 * on the GPU) and evaluates the same 16 flows on the device. */
#define scalar_param 1
#define vector_param 2
struct v_param_t {
  char *name;
  int type;
  union param_value_t {
    struct vec3d vector;
    double scalar;
  } value;
};
struct v_conf_t;
typedef int (*get_v_t)(const struct vec3d *, double, struct vec3d *, struct v_conf_t *vconf);
struct v_conf_t {
  char *name;
  get_v_t fun;
  int n_params;
  struct v_param_t v_params[32];
};
extern struct v_conf_t vn_conf;
extern struct v_conf_t vs_conf;
extern struct v_conf_t vb_conf;
#endif

/* Run-time globals the hot path reads (include/vortex_constants.h:25-78,
 * defaults of src/vortex_constants.c:24-95).  Defined in libov_gpu.so with
 * the reference's defaults; an executable that also links the reference's
 * vortex_constants.o interposes its own definitions, which the library then
 * reads. */
extern double VORTEX_WIDTH;
extern double KAPPA;
extern int global_LIA_only;
extern double global_alpha;
extern double global_alpha_p;
extern double global_dl_max;
extern int global_num_threads;
extern int global_use_mutual_friction;
extern int global_use_BH;
extern double global_BH_resolution;
extern int global_BH_quadtree;
extern double global_BH_grain;
extern int global_hyperfriction;
extern double global_max_curvature_scale;
extern double global_hyperalpha;
/* loop removal (include/vortex_constants.h:41,49-56) */
extern int global_small_loop_cutoff;
extern int global_eliminate_origin_loops;
extern double global_eliminate_loops_origin_cutoff;
extern int global_eliminate_zaxis_loops;
extern double global_eliminate_loops_zaxis_cutoff;
extern int global_eliminate_outer_loops;
extern double global_eliminate_outer_loops_cutoff;

/* ===================================================================== */
/* Part 2: extensions (no reference counterpart)                          */
/* ===================================================================== */

/* status codes */
enum {
  OV_OK = 0,
  OV_ERR_NO_DEVICE = 1,   /* no CUDA device / library built without sm_100a */
  OV_ERR_CUDA = 2,        /* CUDA runtime error */
  OV_ERR_INVALID = 3,     /* bad argument or tangle (broken links, bad sizes) */
  OV_ERR_NONFINITE = 4,   /* NaN/Inf in inputs or results */
  OV_ERR_FLOW = 5,        /* unknown external flow name / missing parameter */
  OV_ERR_TREE_DEPTH = 6,  /* box/BH_grain ratio needs more than 32 tree levels */
  OV_ERR_TIMEOUT = 7,     /* a bounded device wait ran out */
  OV_ERR_NOMEM = 8        /* device allocation failed */
};

/* precision modes */
enum {
  OV_PREC_FP64 = 0,  /* everything in FP64: the reference's arithmetic */
  OV_PREC_MIXED = 1  /* FP32 far field, FP64 positions/local term/near field */
};

/* Select the CUDA device (default 0).  Called implicitly by the first call. */
int ov_init(int device);
int ov_last_error(void);
const char *ov_last_error_message(void);
const char *ov_error_string(int code);
void ov_clear_error(void);

/* precision of subsequent calls (process-wide); default OV_PREC_FP64 */
void ov_set_precision(int mode);
int ov_get_precision(void);
/* 0 (default): the reference's RK4, whose fourth stage advances dt/2
 * (src/vortex_dynamics.c:89); 1: classic RK4 (fourth stage advances dt) */
void ov_set_rk4_classic(int classic);
int ov_get_rk4_classic(void);
/* Mixed form: interactions closer than factor * global_dl_max to the target
 * (segments and cell expansions) are evaluated in FP64 (default 8; segments
 * nearer than 4 times their own length always are). */
void ov_set_mixed_near_factor(double factor);
double ov_get_mixed_near_factor(void);

/* The colinearity cut-off of the segment formula: a segment adds nothing
 * where |cos(R, R') - 1| < eps (the reference's eps = 1e-8,
 * src/tangle.c:505-506, the default).  It makes the velocity discontinuous
 * where a segment's extension passes near a target.  eps = 0 switches it
 * off in the FP64 direct sums and in the adjoint (ov_adjoint_*), for
 * gradient checks against finite differences of a smooth function; the
 * Barnes-Hut walks and the mixed form keep the reference's value.  Not the
 * reference's behaviour when changed.  Captured when a tangle is uploaded. */
void ov_set_colinear_cutoff(double eps);
double ov_get_colinear_cutoff(void);

/* Per-call counters of the last velocity evaluation on this thread. */
typedef struct {
  double interactions;      /* segment-point interactions (direct and P2P) */
  double cell_interactions; /* Barnes-Hut multipole evaluations */
  double cells;             /* octree cells built */
  double eval_ms;           /* device time of the Biot-Savart kernel */
  double build_ms;          /* device time of the tree build */
  double total_ms;          /* device time of the whole evaluation */
} ov_eval_stats;
int ov_get_last_stats(ov_eval_stats *out);

/* ----- device-resident state: upload once, step many times ----- */
typedef struct ov_state ov_state;
ov_state *ov_state_create(void);
void ov_state_destroy(ov_state *s);
/* copy a host tangle (positions, links, status, box, images, vels) in */
int ov_state_upload(ov_state *s, const struct tangle_state *tangle);
/* copy results out; what: bitmask of OV_FIELD_* */
enum {
  OV_FIELD_POS = 1, OV_FIELD_VELS = 2, OV_FIELD_VS = 4, OV_FIELD_TANGENTS = 8,
  OV_FIELD_NORMALS = 16, OV_FIELD_DXI = 32, OV_FIELD_ALL = 63
};
int ov_state_download(ov_state *s, struct tangle_state *tangle, int what);
/* update_tangle (tangents, normals, velocities) on the device state */
int ov_state_update_tangle(ov_state *s, double t);
/* rk4_step on the device state (uses its current vels as k1) */
int ov_state_rk4_step(ov_state *s, double t, double dt);
/* nsteps x (update_tangle + rk4_step), time advancing by dt */
int ov_state_run(ov_state *s, double t0, double dt, int nsteps);
/* ----- one tangle over several ranks (one process per GPU) -----
 * Every rank holds the whole tangle and builds the same tree; rank r of W
 * walks only the targets at key positions [r*c, (r+1)*c) of that tree,
 * c = ceil(active nodes / W), so the Biot-Savart sums, nearly all the work
 * of an evaluation, split W ways.  The sums are exchanged through xbuf, a
 * device buffer of ov_state_shard_bytes(s, W) bytes (6 doubles per key
 * position, rank r's block at r*c*6) that the caller all-gathers in place
 * between begin and end (e.g. ncclAllGather with sendbuff = xbuf + r*c*6,
 * recvbuff = xbuf, count c*6).  Every rank then finishes every node, so all
 * ranks keep identical states and the results equal ov_state_run's bit for
 * bit.  One RK4 step = stages 0..3, each begin / exchange / end:
 *   stage 0: update_tangle at the positions (k1 into vels, vs)
 *   stage q = 1..3: the q-th stage of rk4_step; stage 3 ends with the
 *            combination that advances the positions
 * begin returns once xbuf holds this rank's block; end reads all of xbuf.
 * Needs the Barnes-Hut path (global_use_BH) unless global_LIA_only.  W = 1
 * with xbuf NULL runs the same stages on one GPU.  No counterpart in the
 * reference, which runs a tangle in one process. */
int ov_state_shard(ov_state *s, int rank, int world, void *xbuf, size_t bytes);
size_t ov_state_shard_bytes(ov_state *s, int world);
int ov_state_shard_begin(ov_state *s, int stage, double t, double dt);
int ov_state_shard_end(ov_state *s, int stage, double t, double dt);

/* Biot-Savart velocity (nonlocal + images, no LIA/friction) at arbitrary
 * points from the state's current positions: method 0 = direct sum,
 * 1 = Barnes-Hut.  pts/out: host arrays of 3*npts doubles; skip: per-point
 * node to skip (NULL = none). */
int ov_state_eval_points(ov_state *s, int npts, const double *pts, const int *skip,
                         int method, double *out);

/* Counters accumulated by a state since ov_state_reset_stats:
 * evaluations, segment-point interactions (direct and Barnes-Hut leaves),
 * multipole evaluations, device time of the Biot-Savart kernels and of the
 * tree builds, kernel launches by this library, and the device time of the
 * last ov_state_run (CUDA events on the state's stream). */
typedef struct {
  double evals;
  double interactions;
  double cell_interactions;
  double bs_kernel_ms;
  double bs_launches;
  double build_ms;
  double last_run_ms;
  double launches;
  double n_targets;
  double n_segments;
  double warp_iterations;   /* Barnes-Hut walk: cells visited per warp, summed */
} ov_run_stats;
int ov_state_get_stats(ov_state *s, ov_run_stats *out);
void ov_state_reset_stats(ov_state *s);

/* Direct Biot-Savart velocity (the tangle's own segments plus the boundary
 * image sum, as ov_state_eval_points with method 0) at npts points, for
 * callers that cannot call cudaMalloc: code whose device memory is owned by
 * another framework's allocator, or a loop that must not allocate.  It
 * allocates nothing: inputs and outputs are the caller's device buffers and
 * the scratch (segment table and per-image partial sums) is one file-scope
 * device array of fixed size that every GPU loading this library holds
 * until the process exits.  No counterpart in the reference.
 *   header   host tangle header: only N, box and bimg are read
 *   d_pos    3*N doubles, d_links 2*N ints (forward, reverse), d_status
 *            2*N ints (status, pin wall), all device memory
 *   d_pts    3*npts doubles, d_skip npts ints or NULL (node skipped in the
 *            tangle's own sum), d_out 3*npts doubles, all device memory
 *   stream   a cudaStream_t (NULL: the default stream); the call only
 *            enqueues work on it and returns
 * Limits: N <= OV_NOALLOC_MAX_NODES, npts <= OV_NOALLOC_MAX_POINTS and
 * npts * (1 + bimg.n) <= OV_NOALLOC_MAX_POINT_IMAGES; larger sizes return
 * OV_ERR_INVALID.  The first call on each device looks up the array's device
 * address (cudaGetSymbolAddress) with that device current; make that first
 * call before any stream capture.  All calls share the one array, which
 * keeps the last call's contents: calls whose work overlaps on the GPU (on
 * different streams, or host threads) race.  The looked-up address is kept
 * for the life of the process: after cudaDeviceReset (or with another
 * context made current on that device) it no longer names the array, so do
 * not call this entry point again in that process after such a reset. */
#define OV_NOALLOC_MAX_NODES 131072
#define OV_NOALLOC_MAX_POINTS 131072
#define OV_NOALLOC_MAX_POINT_IMAGES 131072
int ov_direct_points_noalloc(const struct tangle_state *header, const double *d_pos,
                             const int *d_links, const int *d_status, int npts,
                             const double *d_pts, const int *d_skip, double *d_out,
                             void *stream);

/* ----- batched ensembles of independent systems -----
 * Many small open-boundary systems (each a few closed loops) advanced
 * together: the reference runs one tangle per process, so this has no
 * counterpart there.  Every system evolves exactly as a tangle of its own
 * would under update_tangle + rk4_step: its velocity sums only its own
 * segments (direct Biot-Savart, no tree, no images); local induction,
 * external flows, hyperfriction and mutual friction are per node as usual.
 *   all      one tangle_state holding every system's slots, system s in
 *            slots offsets[s] .. offsets[s+1]-1; every link stays inside its
 *            system; all six walls open, no boundary images
 *   offsets  n_systems + 1 non-decreasing slot offsets, offsets[0] = 0,
 *            offsets[n_systems] = all->N
 * The globals and flows are read at create and at every run/update call;
 * ov_set_precision selects FP64 or the mixed form (FP32 beyond the near
 * radius, which here is the near factor times each system's own longest
 * segment).  The Biot-Savart sum of all systems is one persistent kernel
 * per RK4 stage that takes (system, block of targets) work items, largest
 * systems first; ov_batch_run captures one RK4 step in a CUDA graph and
 * replays it. */
typedef struct ov_batch ov_batch;
ov_batch *ov_batch_create(const struct tangle_state *all, int n_systems, const int *offsets);
void ov_batch_destroy(ov_batch *b);
/* one velocity evaluation (update_tangle) at the current positions */
int ov_batch_update(ov_batch *b, double t);
/* nsteps x (update_tangle + rk4_step) at t0, t0 + dt, ..., as one CUDA
 * graph per RK4 step, replayed */
int ov_batch_run(ov_batch *b, double t0, double dt, int nsteps);
/* copy results of every system out (OV_FIELD_* mask) */
int ov_batch_download(ov_batch *b, struct tangle_state *all, int what);
/* Biot-Savart kernel shape: targets per block (64, 128 or 256), sources
 * per shared-memory tile (64, 128 or 256; 0: the mixed form in chain order,
 * whose consecutive segments share end nodes, in tiles of 128) and resident
 * blocks per SM of the persistent grid (0: as many as fit).
 * ov_batch_autotune times the candidates on the batch's own systems and
 * keeps the fastest. */
typedef struct {
  int targets_per_block;
  int sources_per_tile;
  int blocks_per_sm;
  double kernel_ms;   /* device time of one Biot-Savart launch (autotune) */
} ov_batch_tuning;
int ov_batch_set_tuning(ov_batch *b, const ov_batch_tuning *tuning);
int ov_batch_get_tuning(ov_batch *b, ov_batch_tuning *out);
int ov_batch_autotune(ov_batch *b, ov_batch_tuning *out);
/* counters: evaluations and segment-point interactions since creation,
 * device time of the last run, average device time of the Biot-Savart
 * launches of the last RK4 step (or of the last update), kernels per RK4
 * step, and the ensemble's targets, segments and systems */
typedef struct {
  double evals;
  double interactions;
  double last_run_ms;
  double bs_kernel_ms;
  double kernels_per_step;
  double n_targets;
  double n_segments;
  double n_systems;
} ov_batch_stats;
int ov_batch_get_stats(ov_batch *b, ov_batch_stats *out);

/* ----- adjoint of an RK4 trajectory with fixed topology -----
 * Reverse-mode derivatives of the velocity and of nsteps x (update_tangle +
 * rk4_step) with respect to the initial positions and the normal-fluid
 * velocity vector (the "simple" flow of vn_conf, driving mutual friction).
 * The reference has no derivatives; the forward dynamics are its own
 * (update_velocity, src/tangle.c:583-684; rk4_step, src/vortex_dynamics.c:
 * 58-121) with reconnection and remeshing off.  Scope: closed loops of free
 * nodes (EMPTY slots allowed), open boundaries, no images, direct sum (the
 * tree setting is ignored), superfluid and normal-fluid flows "no flow" or
 * "simple".  Precision follows ov_set_precision for the forward velocities;
 * the vector-Jacobian products are FP64.  Positions and cotangents are host
 * arrays of 3*N doubles (slot order); vn is 3 doubles (NULL: keep the
 * current vector, initially vn_conf's).  Branch decisions (hyperfriction
 * threshold, cut-offs) are those of the forward values. */
typedef struct ov_adjoint ov_adjoint;
ov_adjoint *ov_adjoint_create(const struct tangle_state *tangle);
void ov_adjoint_destroy(ov_adjoint *a);
/* velocities at positions x */
int ov_adjoint_velocity(ov_adjoint *a, const double *x, const double *vn, double t, double *v);
/* x_bar = (dv/dx)^T v_bar and vn_bar = (dv/dvn)^T v_bar at positions x */
int ov_adjoint_velocity_vjp(ov_adjoint *a, const double *x, const double *vn, double t,
                            const double *v_bar, double *x_bar, double *vn_bar);
/* nsteps RK4 steps from x0 at t0, positions checkpointed every
 * checkpoint_every steps; x_final may be NULL */
int ov_adjoint_forward(ov_adjoint *a, const double *x0, const double *vn, double t0, double dt,
                       int nsteps, int checkpoint_every, double *x_final);
/* cotangent of the last forward run's final positions -> cotangents of its
 * initial positions and of vn (recomputing each block of steps from its
 * checkpoint, with the vn and precision that forward run used) */
int ov_adjoint_backward(ov_adjoint *a, const double *x_final_bar, double *x0_bar, double *vn_bar);
/* number of completed ov_adjoint_forward runs on a: a caller holding
 * several trajectories of one handle compares it to the value after its
 * own forward run to know whether backward still refers to that run */
unsigned long long ov_adjoint_generation(const ov_adjoint *a);

/* ----- vortex-vortex reconnection with the pair search on the GPU -----
 * The reference's pair loop (reconnect, src/vortex_dynamics.c:216-313)
 * tests all N^2/2 node pairs.  The tests that cannot change during a pass
 * (neither node empty or pinned, not linked, distance after the periodic
 * wrap <= rec_dist, both tangents >= 0.5 long, tangents at an angle above
 * rec_angle) are done here by a GPU grid search in the reference's FP64
 * operations.  tangle->tangents must be current.
 * ov_reconnect_candidates writes up to max_pairs pairs (k, l), k < l, as
 * 2 ints each, in the loop's order (k, then l ascending), and returns how
 * many there are (or -OV_ERR_*).  ov_reconnect_vortices then runs the rest
 * of the loop on the host in that order: the links and sit-out flags
 * (tangle->recalculate) of the pass so far, the approach test with
 * update_velocity of both nodes (direct sum, as the reference), and
 * do_reconnection (src/vortex_dynamics.c:317-364).  Its result is the
 * reference loop's: same links, flags, velocities written and count
 * (returned, or -OV_ERR_*).  Wall reconnections, small-loop removal and
 * domain cleanup stay with the reference's reconnect(), which zeroes
 * tangle->recalculate before them: ov_reconnect_vortices reads the flags
 * as it finds them, so a caller without the wall part zeroes them first. */
int ov_reconnect_candidates(const struct tangle_state *tangle, double rec_dist, double rec_angle,
                            int *pairs, int max_pairs);
int ov_reconnect_vortices(struct tangle_state *tangle, double t, double rec_dist, double rec_angle);

/* In the mixed form (ov_set_precision(OV_PREC_MIXED)) ov_reconnect_vortices
 * takes the approach test's Biot-Savart sums with the FP32 far field and a
 * bound on their error per node; a test whose sign that bound leaves open
 * is taken again with FP64 sums, so links, flags and count are the FP64
 * form's, and the velocities it writes carry the mixed form's error.  The
 * environment variable OV_RECONNECT_MARGIN_SCALE multiplies that margin (a
 * huge value sends every test to the FP64 re-check; for tests).
 * Counters of the last ov_reconnect_vortices call on this thread: */
typedef struct {
  int candidates;     /* pairs that passed the static tests */
  int tested;         /* approach tests taken */
  int nodes_summed;   /* nodes whose sums came from a batched direct sum */
  int fp64_rechecks;  /* mixed form: tests taken again with FP64 sums */
  int reconnections;
  double search_s;    /* host seconds: upload and the GPU pair search */
  double sums_s;      /* host seconds in the batched (and re-check) sums */
  double total_s;     /* host seconds of the whole call */
} ov_reconnect_stats;
int ov_reconnect_get_stats(ov_reconnect_stats *out);

/* ----- remesh and periodic wrap-around -----
 * ov_remesh replaces remesh (src/tangle.c:824-873, include/tangle.h:155):
 * the reference's slot-order loop that removes a node when a segment next
 * to it is shorter than min_dist (merging it into that neighbour,
 * remove_point) and the two together shorter than max_dist, and adds a
 * node after a node whose forward segment is longer than max_dist
 * (add_point), then enforce_boundaries if it added any.  Same nodes
 * removed and added, same slots (search_next_free), same links; positions,
 * tangents, normals and dxi as the reference's to rounding.  The tangle's
 * dxi, tangents and normals must be current on entry (main.c computes them
 * right before remesh) and are current on return.  New nodes take EMPTY
 * slots; with none left, expand (the reference's expand_tangle) doubles
 * the tangle, or without it the call fails with OV_ERR_INVALID after the
 * changes made so far.  Returns the number of nodes removed plus added,
 * or -OV_ERR_*.
 * ov_enforce_boundaries replaces enforce_boundaries (src/tangle.c:796-819,
 * include/tangle.h:118): every node outside the box through a periodic
 * face moves by box lengths until it is inside.  Returns the number of
 * nodes moved, or -OV_ERR_*. */
typedef void (*ov_expand_fn)(struct tangle_state *tangle, size_t n);
int ov_remesh(struct tangle_state *tangle, double min_dist, double max_dist, ov_expand_fn expand);
int ov_enforce_boundaries(struct tangle_state *tangle);

/* ov_eliminate_small_loops replaces eliminate_small_loops
 * (src/tangle.c:876-943, include/tangle.h:156): every closed loop or pinned
 * line with fewer than loop_length + 1 nodes is emptied and unlinked, and
 * before that, when global_eliminate_origin_loops / _zaxis_loops /
 * _outer_loops are set, every loop lying wholly within the origin cut-off,
 * within the z-axis cut-off or beyond the outer cut-off
 * (src/tangle.c:945-1015).  The nodes removed and links left are the
 * reference's; tangle->recalculate, which the reference uses as visit marks,
 * is not written.  Returns the number of vortices removed, or -OV_ERR_*. */
int ov_eliminate_small_loops(struct tangle_state *tangle, int loop_length);

/* ----- frames -----
 * Text frames (OV_FRAME_TEXT) are the reference's save_tangle files
 * (src/vortex_utils.c:308-345, include/vortex_utils.h), byte for byte:
 * ov_save_tangle replaces save_tangle (without its "saving frame" line on
 * stdout); the rows are formatted on all host cores.
 * Binary frames (OV_FRAME_BINARY) add the simulation time, which text
 * frames lack, and hold every slot as it is, little-endian:
 *   struct ov_frame_header (128 bytes), then in slot order
 *   vnodes, vels, tangents, normals   N x 3 doubles each
 *   dxi                               N doubles
 *   connections                       N x (forward, reverse) int32
 *   status                            N x (status, pin_wall) int32
 * (arrays the tangle does not have are written as zeros).
 * ov_state_save_frame takes the frame from a device-resident state and
 * returns at once: the state's arrays are copied on the device in its
 * stream order, so later steps do not change the frame, and the file is
 * written by a background thread.  A state's next frame waits for its
 * previous one; ov_frame_wait waits for every pending write and returns
 * the first failure.  ov_state_destroy waits for the state's frame; do not
 * destroy a state while another thread is in ov_frame_wait.
 * ov_load_frame reads a binary frame into a tangle of exactly the frame's
 * slot count (ov_frame_info tells it), box and walls included. */
enum { OV_FRAME_TEXT = 0, OV_FRAME_BINARY = 1 };
typedef struct ov_frame_header {
  char magic[8]; /* "OVFRAME" */
  int32_t version; /* 1 */
  int32_t n;       /* slots */
  double time;     /* simulation time of the frame */
  double box_lo[3], box_hi[3];
  int32_t wall[6];
  int32_t reserved[8];
} ov_frame_header;
int ov_save_tangle(const struct tangle_state *tangle, const char *filename);
int ov_save_frame(const struct tangle_state *tangle, const char *filename, double time, int format);
int ov_state_save_frame(ov_state *s, const char *filename, double time, int format);
int ov_frame_wait(void);
int ov_frame_info(const char *filename, int *n, double *time);
int ov_load_frame(const char *filename, struct tangle_state *tangle, double *time);

/* Sustained FMA throughput of this GPU in TFLOP/s (2 flops per FMA),
 * fp64 = 0 for FP32, 1 for FP64: the roofline denominator. */
int ov_measure_fma_peak(int fp64, double *tflops);

/* Accuracy of the FP64 reciprocal square root and reciprocal the direct
 * sum uses in place of IEEE sqrt and division (hardware approximation plus
 * two Newton-Raphson steps): the largest differences from 1/sqrt(x) and
 * 1/x computed with IEEE operations on the device, in ulps, over
 * x = 2^(e/64), e in [-8192, 8192).  No counterpart in the reference. */
int ov_check_fast_math(double *rsqrt_ulps, double *rcp_ulps);

#ifdef __cplusplus
}
#endif
#endif /* OPENVORT_B200_H */
