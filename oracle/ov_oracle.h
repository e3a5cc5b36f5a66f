/*
 * ov_oracle.h - CPU restatement of OpenVort's Schwarz vortex-filament
 * velocity + RK4 path.  TEST INFRASTRUCTURE ONLY: the checker that the CUDA
 * product is compared against.  Nothing in the product links or calls this.
 *
 * Parity pinned against the reference compiled from its own sources
 * (oracle/_ref, built by oracle/Makefile) and against golden vectors the
 * reference produced (tests/golden/).
 *
 * Layout: plain arrays indexed by node slot, like the reference's
 * struct tangle_state (include/tangle.h:82-106 of the reference).
 */
#ifndef OV_ORACLE_H
#define OV_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* node status values, as node_status_t in the reference (include/tangle.h:28-33) */
enum { OVO_EMPTY = -1, OVO_FREE = 0, OVO_PINNED = 1, OVO_PINNED_SLIP = 2 };
/* wall types, as wall_type (include/vec3_maths.h:31) */
enum { OVO_WALL_OPEN = 0, OVO_WALL_PERIODIC = 1, OVO_WALL_MIRROR = 2 };

/* external flow kinds, one per entry of v_confs[] in the reference
 * (src/external_velocity.c:85-170), in that table's order */
enum {
  OVO_FLOW_NONE = 0, OVO_FLOW_SPHERICAL, OVO_FLOW_SIMPLE, OVO_FLOW_SPHERICAL_SIMPLE,
  OVO_FLOW_CYLINDRICAL, OVO_FLOW_OSCILLATING, OVO_FLOW_OSCILLATING_SLIT,
  OVO_FLOW_COSCOS, OVO_FLOW_COSCOS_DIVFREE, OVO_FLOW_COS_DIVFREE,
  OVO_FLOW_SIMPLE_SHEAR, OVO_FLOW_ROTOSC, OVO_FLOW_DG, OVO_FLOW_ROTOSC_BOUNDARY,
  OVO_FLOW_CONST_ACCEL, OVO_FLOW_PARABOLIC, OVO_FLOW_COUNT
};

/* A flow: kind + up to 4 scalars + up to 2 vectors.  Slot meaning per kind is
 * documented in ov_oracle.c (ovo_flow_eval). */
typedef struct {
  int kind;
  double s[4];
  double v[2][3];
} ovo_flow;

typedef struct {
  int n;               /* number of slots */
  const double *pos;   /* 3n */
  const int *fwd;      /* n, -1 = none */
  const int *rev;      /* n */
  const int *status;   /* n, OVO_* */
  const int *pin_wall; /* n, boundary_faces or -1 */
  double lo[3], hi[3]; /* domain box */
  int wall[6];         /* X_L, X_H, Y_L, Y_H, Z_L, Z_H */
  int n_img;
  const int *img;      /* 4 ints per image: shift x,y,z, reflect face (-1 none) */
} ovo_tangle;

typedef struct {
  double kappa, core_a;
  int lia_only;
  int use_bh, bh_quadtree;
  double bh_theta, bh_grain;
  int use_mf;
  double alpha, alpha_p;
  int hyperfriction;
  double max_curv_scale, hyperalpha, dl_max;
  int rk4_classic;     /* 0: reference stage-4 half step (src/vortex_dynamics.c:89) */
  ovo_flow vn, vs, vb;
} ovo_params;

/* dxi + tangents + normals (update_tangents_normals, src/tangle.c:704-727) */
void ovo_tangents_normals(const ovo_tangle *t, double *dxi, double *tangents,
                          double *normals);

/* per-node velocities (update_velocities, src/tangle.c:583-702); needs
 * tangents/normals.  vels, vs: 3n outputs (EMPTY slots untouched). */
void ovo_velocities(const ovo_tangle *t, const ovo_params *p, double time,
                    const double *tangents, const double *normals, double *vels,
                    double *vs);

/* velocity of all segments at points (calculate_vs, src/tangle.c:553-581) */
void ovo_segments_at(const ovo_tangle *t, const ovo_params *p, int npts,
                     const double *pts, const int *skip, double *out);

/* Barnes-Hut query at points (octree_build + octree_get_vs, src/octree.c) */
void ovo_bh_at(const ovo_tangle *t, const ovo_params *p, int npts,
               const double *pts, const int *skip, double *out);

/* One RK4 step in place (rk4_step, src/vortex_dynamics.c:58-121).
 * pos is updated; vels_k1 must hold the velocities at the current positions. */
void ovo_rk4_step(const ovo_tangle *t, const ovo_params *p, double time,
                  double dt, double *pos, const double *vels_k1);

/* convenience: tangents/normals + velocities (update_tangle, include/tangle.h:160) */
void ovo_update_tangle(const ovo_tangle *t, const ovo_params *p, double time,
                       double *dxi, double *tangents, double *normals,
                       double *vels, double *vs);

#ifdef __cplusplus
}
#endif
#endif
