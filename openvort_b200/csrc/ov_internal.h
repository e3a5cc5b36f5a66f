// ov_internal.h - host-side internals shared by the translation units of
// libov_gpu.so: the device state behind ov_state, the Barnes-Hut tree, the
// error channel and the kernel launchers.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>
#include <string>

#include "openvort_b200.h"
#include "ov_device.cuh"

// ---------------------------------------------------------------- errors
void ov_set_error(int code, const char* fmt, ...);
bool ov_cuda_ok(cudaError_t e, const char* what);
#define OV_TRY_CUDA(expr)                          \
  do {                                             \
    if (!ov_cuda_ok((expr), #expr)) return false;  \
  } while (0)

// ---------------------------------------------------------------- buffers
// Grow-only device buffer.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  bool reserve(size_t n);
  void release();
  template <class T> T* as() const { return static_cast<T*>(p); }
};

// ---------------------------------------------------------------- BH tree
// Octree cell kinds (what the walk does with a cell it reaches):
//   CELL_LEAF1    : a single node (N == 1): its segment, inline in the record
//   CELL_LEAFN    : several nodes in a box below BH_grain: direct sum over the
//                   cell's node range, no opening test
//   CELL_OPEN     : opening test; on failure descend into the children
//   CELL_OPEN_P2P : opening test; on failure direct sum over the cell's nodes
//                   (a chain of single-child cells ending in a grain leaf)
//   CELL_OPEN_ZERO: opening test; on failure nothing (unsplit, or every node
//                   dropped from the children, src/octree.c:104,118-127)
enum { CELL_LEAF1 = 0, CELL_LEAFN = 1, CELL_OPEN = 2, CELL_OPEN_P2P = 3, CELL_OPEN_ZERO = 4 };

// One cell in depth-first preorder, one 128-byte line.  Children of cell c
// start at c + 1; the first cell after c's subtree is `skip`.
//   bytes   0-15  : a, b, skip, meta = kind | level_top << 8 | level_bot << 16
//                   LEAF1: a = node slot, b = forward slot
//                   LEAFN: a = first sorted node, b = node count
//                   OPEN*: a = FP32 m21 (bit pattern), b = FP32 rounding
//                   margin of the opening test (bit pattern, mac_margin)
//                   level_top..level_bot: the octree levels the (chain of)
//                   cell(s) spans; children start at level_bot + 1
//   bytes  16-23  : thr, the opening test passes iff the reference-wrapped
//                   squared distance to the centre of mass is >= thr
//   bytes  24-47  : x = centre of mass (LEAF1: segment start r1)
//   bytes  48-71  : y = kappa/4pi * total circulation (LEAF1: wrapped r2)
//   bytes  72-103 : kappa/4pi * (m21, m02, m12, m22), FP64
//   bytes 104-127 : FP32 circulation and m02, m12, m22 (the mixed form reads
//                   bytes 0-47 and 104-127 only)
// Node ranges of every cell (first sorted node, count) are in a side array.
struct __align__(128) Cell {
  int a, b, skip, meta;
  double thr;
  double x[3];
  double y[3];
  double m[4];
  float f_g[3];
  float f_m02, f_m12, f_m22;
};
static_assert(sizeof(Cell) == 128, "cell record is one 128-byte line");
// the walk loads these fields with vector loads of the given width
static_assert(offsetof(Cell, a) % 16 == 0, "int4 header load");
static_assert(offsetof(Cell, thr) % 16 == 0, "double2 (thr, x0) load");
static_assert(offsetof(Cell, x) % 16 == 8 && (offsetof(Cell, x) + 8) % 16 == 0, "double2 (x1, x2) load");
static_assert(offsetof(Cell, f_g) % 8 == 0 && offsetof(Cell, f_m12) % 8 == 0, "float2 loads");
__host__ __device__ __forceinline__ int cell_kind(int meta) { return meta & 7; }
__host__ __device__ __forceinline__ int cell_ltop(int meta) { return (meta >> 8) & 63; }
__host__ __device__ __forceinline__ int cell_lbot(int meta) { return (meta >> 16) & 63; }

struct OvTree {
  int n_nodes = 0;      // active (non-EMPTY) nodes
  int n_drop_root = 0;  // active nodes outside the root box (sorted last)
  int n_cells = 0;
  int built = 0;
  double theta = 0;     // theta used for thr
  OvParams P;           // parameters at build time
  DevBuf keys, keys_alt, vals, vals_alt, stop, hist;   // sort
  DevBuf perm;          // sorted index -> slot
  DevBuf bnode;         // binary radix tree nodes
  DevBuf cstart_cnt, cbase, cell_of;   // preorder bookkeeping
  DevBuf cells, cell_lm, cell_range;   // cell records, max box side, node range per cell
  DevBuf nodes64;       // per sorted node: r1 (3), r2 wrapped (3)
  DevBuf nodeids;       // per sorted node: slot, forward slot
  DevBuf nodes32;       // per sorted node: r1 - cell-free origin (FP32 not used yet)
  DevBuf counters;      // device counters (interactions, cells visited)
  DevBuf scratch;
  DevBuf scan_part;     // block sums of the exclusive scans
  DevBuf mom_part;      // per-chunk partial moments of the largest cells
  DevBuf walk_order;    // the walk's target list when nodes lie outside the root box
  // the multi-image walk's groups of 32 targets by decreasing time in the
  // last walk (wvals after the sort), their times, and the sort's buffers
  DevBuf warp_cost, wkeys, wkeys2, wvals, wvals2, whist, wscan;
  int n_perm_warps = 0;   // groups the order in wvals covers (0: none yet)
};

// ---------------------------------------------------------------- state
struct ov_state_impl {
  int cap = 0;          // slot capacity of the device arrays
  int n = 0;            // slots in use
  OvParams P;           // captured at upload / call time
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
  // slot-indexed (AoS, 3 doubles per vector, as struct vec3d)
  DevBuf pos, links, status, dxi, tan, nrm, vels, vs;
  // RK4 scratch
  DevBuf pos0, spos, sdxi, stan, snrm, svs, k2, k3, k4;
  // Biot-Savart outputs: primary sum and image sum per slot
  DevBuf v_nl, v_img;
  // direct-sum per-image partials and segment table
  DevBuf img_part, seg64, segid;
  // error flag written by kernels (bounded waits, broken links)
  DevBuf dflag;
  OvTree tree;
  double t_last = 0;
  // accumulated over evaluations since the last reset (ov_state_get_stats)
  double acc_evals = 0, acc_inter = 0, acc_cells = 0, acc_bs_ms = 0, acc_bs_launches = 0;
  double acc_warp_iter = 0;
  double acc_build_ms = 0, last_run_ms = 0;
  long long launches_at_reset = 0;
  int n_targets = 0, n_segments = 0;
  cudaEvent_t ev_run0 = nullptr, ev_run1 = nullptr;
  int walls[6] = {0, 0, 0, 0, 0, 0};   // box.wall of the uploaded tangle
  void* frames = nullptr;              // frame snapshot buffers (ov_frames.cu)
  // one tangle over several ranks (ov_state_shard): this rank's share of
  // the targets, the exchange buffer, and the counters of the walk between
  // ov_state_shard_begin and ov_state_shard_end
  int n_active = 0;                    // non-EMPTY slots of the upload
  int shard_rank = 0, shard_world = 1;
  double* xbuf = nullptr;              // the caller's, or xown's when world is 1
  size_t xbytes = 0;
  DevBuf xown;
  double shard_inter = 0, shard_cells = 0, shard_warp_iter = 0;
};

// the implementation behind a public ov_state handle
ov_state_impl* ov_state_impl_of(ov_state* s);
// waits for and frees a state's frame buffers
void ov_frames_release(ov_state_impl* s);

// ---------------------------------------------------------------- launchers
// geometry: dxi, tangents, normals of all slots (pos/links/status -> dxi,tan,nrm)
bool ov_geometry(ov_state_impl* s, const double* pos, double* dxi, double* tan, double* nrm);
// velocities at positions pos with tangents/normals -> vels, vs
bool ov_velocities(ov_state_impl* s, double t, const double* pos, const double* dxi,
                   const double* tan, const double* nrm, double* vels, double* vs,
                   OvTree* external_tree);
// one RK4 step on the state's pos using the state's vels as k1
bool ov_rk4(ov_state_impl* s, double t, double dt, int classic);
// its pieces: stage q = 1..3 positions into spos, and the final combination
bool ov_rk4_stage_positions(ov_state_impl* s, int q, double dt, int classic);
bool ov_rk4_combine(ov_state_impl* s, double dt);
bool ov_euler(ov_state_impl* s, double dt);

// tree over the positions pos (slot-indexed); fills tree
bool ov_tree_build(ov_state_impl* s, const double* pos, OvTree* tree);
void ov_tree_release(OvTree* tree);
// Barnes-Hut nonlocal + image sums for every active node -> v_nl, v_img
// own_tree: the tree was built from `pos` (targets in its key order); then
// only the targets at key positions [k0, k0 + k_count) are evaluated
// (k_count < 0: all of them)
bool ov_tree_walk_nodes(ov_state_impl* s, OvTree* tree, const double* pos, bool own_tree,
                        double* v_nl, double* v_img, int k0 = 0, int k_count = -1);
// sharded evaluations: v_nl, v_img of the targets at key positions
// [k0, k0 + count) into xbuf (6 doubles per key position), and back from
// xbuf for every active node; xcap: doubles in xbuf
bool ov_shard_pack(ov_state_impl* s, int k0, int count, double* xbuf, size_t xcap);
bool ov_shard_unpack(ov_state_impl* s, const double* xbuf, size_t xcap);
// Barnes-Hut sums at arbitrary points (device arrays): out_nl = the tangle's
// own sum (skip per point), out_img = the image sum (nullptr: no images)
bool ov_tree_walk_points(ov_state_impl* s, OvTree* tree, int npts, const double* pts,
                         const int* skip, double theta, double* out_nl, double* out_img);

// stable LSD radix sort of 64-bit keys with int values (ov_tree.cu); the
// result ends in (ka, va), (kb, vb) are scratch of the same sizes
bool ov_radix_sort_u64(uint64_t* ka, int* va, uint64_t* kb, int* vb, int n, DevBuf& hist, DevBuf& scan_part,
                       cudaStream_t st);
// direct sums for all nodes -> v_nl, v_img
bool ov_direct_nodes(ov_state_impl* s, const double* pos, double* v_nl, double* v_img);
// direct sums at arbitrary points (device arrays), sources = all segments or
// the slot list `only`: out_nl = the tangle's own sum, out_img = image sum
// (nullptr: no images)
bool ov_direct_points(ov_state_impl* s, const double* pos, int npts, const double* pts,
                      const int* skip, const int* only, int n_only, double* out_nl,
                      double* out_img);
// mixed-form direct sums at points (tangle and images, every segment), with
// out_bound[i] bounding |mixed - FP64| of out_nl + out_img at point i
bool ov_direct_points_bounded(ov_state_impl* s, const double* pos, int npts, const double* pts,
                              const int* skip, double* out_nl, double* out_img, double* out_bound);
// direct point query on caller-provided scratch (see ov_direct.cu)
bool ov_direct_points_scratch(cudaStream_t st, const OvParams& P, const double* pos,
                              const int2* links, const int2* status, int n, int npts,
                              const double* pts, const int* skip, double* seg, int* fwd,
                              double* part, double* out, double* img);
// s->seg64 / s->segid: r1 and the wrapped r2 of every slot's forward
// segment at positions pos, and the forward slot (-1: no segment)
bool ov_segment_table(ov_state_impl* s, const double* pos);
// out = a + b for n vectors of 3 doubles (device)
bool ov_add3(cudaStream_t st, const double* a, const double* b, double* out, int n);

// epilogue: LIA + external + v_nl + v_img + hyperfriction + mutual friction
// for slots k0 <= k < k1
bool ov_epilogue(ov_state_impl* s, double t, const double* pos, const double* tan,
                 const double* nrm, const double* v_nl, const double* v_img,
                 double* vels, double* vs, int k0, int k1);

bool ov_state_reserve(ov_state_impl* s, int n);

// Launches only, no host synchronisation (CUDA-graph capturable); link and
// finiteness errors accumulate in *flag (bit 0 broken links, bit 1
// non-finite velocity), read back later with ov_flag_status.
bool ov_launch_geometry(cudaStream_t st, const OvParams& P, const int2* links, const int2* status,
                        const double* pos, double* dxi, double* tan, double* nrm, int n, int* flag);
// the same for the slots idx[0 .. n-1] only (dxi of all of them first, then
// the two tangent passes); the other slots' values are read as stored
bool ov_launch_geometry_list(cudaStream_t st, const OvParams& P, const int2* links, const int2* status,
                             const double* pos, double* dxi, double* tan, double* nrm, const int* idx, int n,
                             int* flag);
// epilogue at time t0 + *t_dev (t_dev may be null: time t0)
bool ov_launch_epilogue(cudaStream_t st, const OvParams& P, const int2* links, const int2* status,
                        const double* t_dev, double t0, const double* pos, const double* tan,
                        const double* nrm, const double* v_nl, const double* v_img, double* vels,
                        double* vs, int k0, int k1, int* flag);
// the epilogue of the slots idx[0 .. count-1] at time t0
bool ov_launch_epilogue_list(cudaStream_t st, const OvParams& P, const int2* links, const int2* status,
                             double t0, const double* pos, const double* tan, const double* nrm,
                             const double* v_nl, const double* v_img, double* vels, double* vs,
                             const int* idx, int count, int* flag);
bool ov_launch_euler(cudaStream_t st, const int2* status, const double* x0, const double* v,
                     double h, double* xs, int n);
bool ov_launch_rk4_combine(cudaStream_t st, const int2* status, const double* k1, const double* k2,
                           const double* k3, const double* k4, double dt, double* x, int n);
// error for flag bits h (false and the error set when any bit is set)
bool ov_flag_status(int h, const char* where);

// device selection on first use; the tangle's structure, positions and
// parameters (globals, flows) into s; fields of s back into the tangle
bool ov_ensure_init();
bool ov_upload_tangle(ov_state_impl* s, const tangle_state* t);
bool ov_download_fields(ov_state_impl* s, tangle_state* t, int what);

// per-thread statistics of the last evaluation
struct OvStatsAcc {
  double interactions, cell_interactions, cells, eval_ms, build_ms, total_ms, warp_iterations;
};
OvStatsAcc& ov_stats_tls();

// kernel launches issued by this library (all threads)
void ov_note_launch(int n);
long long ov_launches();
#define OV_LAUNCHED() ov_note_launch(1)
