/*
 * Test-infrastructure harness around the UNMODIFIED OpenVort reference C.
 *
 * This file is compiled together with the reference's own sources
 * (src/tangle.c, src/octree.c, src/vortex_dynamics.c, ... read in place from
 * the reference checkout) into oracle/_ref/libov_ref.so by oracle/Makefile.
 * It only marshals arrays in and out of `struct tangle_state` and selects the
 * boundary-image table and external-flow configurations by name, which the
 * reference normally does in src/configuration.c:299-392 (not buildable here:
 * libconfig is absent).  The physics is entirely the reference's.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this library; the product never does.
 */
#include <stdlib.h>
#include <string.h>

#include "external_velocity.h"
#include "octree.h"
#include "tangle.h"
#include "vec3_maths.h"
#include "vortex_constants.h"
#include "vortex_dynamics.h"

struct tangle_state *refh_new(int n) {
  struct tangle_state *t = (struct tangle_state *)malloc(sizeof(*t));
  create_tangle(t, (size_t)n);
  return t;
}

void refh_free(struct tangle_state *t) {
  free_tangle(t);
  free(t);
}

/* Copy node data in.  status: -1 EMPTY, 0 FREE, 1 PINNED, 2 PINNED_SLIP. */
void refh_load(struct tangle_state *t, int n, const double *pos,
               const int *fwd, const int *rev, const int *status,
               const int *pin_wall, const double *vels) {
  for (int k = 0; k < n; ++k) {
    for (int c = 0; c < 3; ++c) {
      t->vnodes[k].p[c] = pos[3 * k + c];
      t->vels[k].p[c] = vels ? vels[3 * k + c] : 0.0;
    }
    t->connections[k].forward = fwd[k];
    t->connections[k].reverse = rev[k];
    t->status[k].status = (node_status_t)status[k];
    t->status[k].pin_wall = (boundary_faces)pin_wall[k];
  }
  t->next_free = 0;
  t->total_free = 0;
}

static const struct boundary_images *bimg_by_name(const char *name) {
  if (!strcmp(name, "open")) return &open_boundaries;
  if (!strcmp(name, "periodic-6")) return &periodic_6;
  if (!strcmp(name, "periodic-18")) return &periodic_18;
  if (!strcmp(name, "periodic-26")) return &periodic_26;
  if (!strcmp(name, "periodic-z-open-xy")) return &periodic_z_open_xy;
  if (!strcmp(name, "wall-1-open")) return &wall_1_open;
  if (!strcmp(name, "wall-1-18")) return &wall_1_18;
  if (!strcmp(name, "wall-1-26")) return &wall_1_26;
  if (!strcmp(name, "wall-2-4")) return &wall_2_4;
  if (!strcmp(name, "wall-2-2")) return &wall_2_2;
  if (!strcmp(name, "wall-2-26")) return &wall_2_26;
  if (!strcmp(name, "channel-z")) return &channel_z;
  return NULL;
}

/* walls: 6 ints in boundary_faces order (0 open, 1 periodic, 2 mirror). */
int refh_set_box(struct tangle_state *t, const double *lo, const double *hi,
                 const int *walls, const char *bimg_name) {
  const struct boundary_images *b = bimg_by_name(bimg_name);
  if (!b) return -1;
  for (int c = 0; c < 3; ++c) {
    t->box.bottom_left_back.p[c] = lo[c];
    t->box.top_right_front.p[c] = hi[c];
  }
  for (int f = 0; f < 6; ++f) t->box.wall[f] = (wall_type)walls[f];
  t->bimg = *b;
  return 0;
}

/* which: 0 = vn_conf, 1 = vs_conf, 2 = vb_conf.  Parameters are given as
 * (name, 3 doubles) pairs; scalars use the first double. */
int refh_set_flow(int which, const char *name, int nparams,
                  const char **pnames, const double *pvals) {
  struct v_conf_t *dst = which == 0 ? &vn_conf : which == 1 ? &vs_conf : &vb_conf;
  for (int k = 0; v_confs[k].fun; ++k) {
    if (strcmp(v_confs[k].name, name)) continue;
    *dst = v_confs[k];
    for (int p = 0; p < nparams; ++p) {
      for (int q = 0; q < dst->n_params; ++q) {
        if (!dst->v_params[q].name || strcmp(dst->v_params[q].name, pnames[p]))
          continue;
        if (dst->v_params[q].type == vector_param)
          dst->v_params[q].value.vector = vec3(pvals[3 * p], pvals[3 * p + 1], pvals[3 * p + 2]);
        else
          dst->v_params[q].value.scalar = pvals[3 * p];
      }
    }
    return 0;
  }
  return -1;
}

void refh_get(const struct tangle_state *t, int n, double *pos, double *vels,
              double *vs, double *tangents, double *normals, double *dxi) {
  for (int k = 0; k < n; ++k) {
    for (int c = 0; c < 3; ++c) {
      if (pos) pos[3 * k + c] = t->vnodes[k].p[c];
      if (vels) vels[3 * k + c] = t->vels[k].p[c];
      if (vs) vs[3 * k + c] = t->vs[k].p[c];
      if (tangents) tangents[3 * k + c] = t->tangents[k].p[c];
      if (normals) normals[3 * k + c] = t->normals[k].p[c];
    }
    if (dxi) dxi[k] = t->dxi[k];
  }
}

void refh_update_tangle(struct tangle_state *t, double time) {
  update_tangle(t, time);
}

void refh_update_tangents_normals(struct tangle_state *t) {
  update_tangents_normals(t);
}

void refh_update_velocities(struct tangle_state *t, double time) {
  update_velocities(t, time, NULL);
}

void refh_rk4_step(struct tangle_state *t, double time, double dt) {
  rk4_step(t, time, dt);
}

/* velocity of the tangle's segments at arbitrary points (calculate_vs) */
void refh_calculate_vs(struct tangle_state *t, int npts, const double *pts,
                       const int *skip, double *out) {
  for (int i = 0; i < npts; ++i) {
    struct vec3d r = vec3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
    struct vec3d v = calculate_vs(t, r, skip ? skip[i] : -1);
    for (int c = 0; c < 3; ++c) out[3 * i + c] = v.p[c];
  }
}

/* Barnes-Hut query through the reference octree at arbitrary points */
void refh_octree_vs(struct tangle_state *t, int npts, const double *pts,
                    const int *skip, double theta, double *out) {
  struct octree *tree = octree_build(t, global_BH_quadtree);
  for (int i = 0; i < npts; ++i) {
    struct vec3d r = vec3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
    struct vec3d v;
    octree_get_vs(tree, &r, theta, &v, skip ? skip[i] : -1);
    for (int c = 0; c < 3; ++c) out[3 * i + c] = v.p[c];
  }
  octree_destroy(tree);
}

/* CPU-baseline sample: the reference's per-evaluation work on a sample of
 * targets.  Times (seconds) update_tangents_normals over the whole tangle,
 * octree_build over the whole tangle (when global_use_BH), and
 * update_velocity for the m listed nodes in the reference's own OpenMP loop
 * (src/tangle.c:693-699) with global_num_threads threads. */
#include <omp.h>
#include <time.h>
static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

void refh_sample_eval(struct tangle_state *t, double time, const int *idx, int m,
                      double *t_geom, double *t_build, double *t_nodes) {
  double a = now_s();
  update_tangents_normals(t);
  double b = now_s();
  struct octree *tree = global_use_BH ? octree_build(t, global_BH_quadtree) : NULL;
  double c = now_s();
  int i;
#pragma omp parallel private(i) num_threads(global_num_threads)
  {
#pragma omp for
    for (i = 0; i < m; ++i) update_velocity(t, idx[i], time, tree);
  }
  double d = now_s();
  if (tree) octree_destroy(tree);
  *t_geom = b - a;
  *t_build = c - b;
  *t_nodes = d - c;
}

/* The reference's superfluid velocity vs (src/tangle.c:583-637: local term,
 * external flow, Biot-Savart sum and image sum) at the m listed nodes, with
 * its own octree when use_tree (built here, global_BH_resolution) or its
 * direct sum otherwise; dxi, tangents and normals must be current.  Writes
 * 3 m doubles.  Returns the seconds of the tree build in *t_build. */
void refh_sample_vs(struct tangle_state *t, double time, const int *idx, int m, int use_tree,
                    double *out, double *t_build) {
  const int keep = global_use_BH;
  global_use_BH = use_tree;
  double a = now_s();
  struct octree *tree = use_tree ? octree_build(t, global_BH_quadtree) : NULL;
  *t_build = now_s() - a;
  int i;
#pragma omp parallel private(i) num_threads(global_num_threads)
  {
#pragma omp for
    for (i = 0; i < m; ++i) {
      update_velocity(t, idx[i], time, tree);
      for (int c = 0; c < 3; ++c) out[3 * i + c] = t->vs[idx[i]].p[c];
    }
  }
  if (tree) octree_destroy(tree);
  global_use_BH = keep;
}
