/*
 * Test infrastructure: the reference's own main loop (src/main.c:77-118,
 * without configuration parsing, frame output and vortex injection) as a
 * program, built twice by oracle/Makefile from the reference's sources:
 *
 *   _ref/ov_linked_ref  all of the reference's sources, unmodified
 *   _ref/ov_linked_gpu  the same sources with the hot-path functions renamed
 *                       in src/tangle.c and src/vortex_dynamics.c and
 *                       src/octree.c left out, linked against libov_gpu.so:
 *                       the integration recipe this library documents, so
 *                       update_tangle, rk4_step and reconnect's
 *                       update_velocity resolve to the GPU library
 *
 *   ov_linked_{ref,gpu} <in.bin> <out.bin>
 *
 * in.bin (little-endian): int32 N, steps, use_bh; double theta, dt,
 * rec_dist, rec_angle, dl_min, dl_max, core_a, alpha, alpha_p, vn[3],
 * lo[3], hi[3]; int32 walls[6]; char bimg[32]; then N x double[3]
 * positions and N x int32 each of forward, reverse, status, pin wall.
 * out.bin: int32 N, reconnections; N x double[3] positions; N x int32 each
 * of forward, reverse, status.  Mutual friction on with vn as the "simple"
 * normal-fluid flow, no superfluid flow; hyperfriction on.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "external_velocity.h"
#include "tangle.h"
#include "vortex_constants.h"
#include "vortex_dynamics.h"

int refh_set_box(struct tangle_state *t, const double *lo, const double *hi, const int *walls,
                 const char *bimg_name);
int refh_set_flow(int which, const char *name, int nparams, const char **pnames,
                  const double *pvals);

#define READ(ptr, size, count)                                         \
  do {                                                                 \
    if (fread((ptr), (size), (count), f) != (size_t)(count)) {         \
      fprintf(stderr, "short read of %s\n", argv[1]);                  \
      return 2;                                                        \
    }                                                                  \
  } while (0)

int main(int argc, char **argv) {
  if (argc != 3) {
    fprintf(stderr, "usage: %s in.bin out.bin\n", argv[0]);
    return 2;
  }
  FILE *f = fopen(argv[1], "rb");
  if (!f) {
    perror(argv[1]);
    return 2;
  }
  int hdr[3];
  double prm[18];
  int walls[6];
  char bimg[33] = {0};
  READ(hdr, sizeof(int), 3);
  READ(prm, sizeof(double), 18);
  READ(walls, sizeof(int), 6);
  READ(bimg, 1, 32);
  const int n = hdr[0], steps = hdr[1];
  struct tangle_state *t = (struct tangle_state *)malloc(sizeof(*t));
  create_tangle(t, (size_t)n);
  double *pos = (double *)malloc(sizeof(double) * 3 * n);
  int *iv = (int *)malloc(sizeof(int) * 4 * n);
  READ(pos, sizeof(double), 3 * n);
  READ(iv, sizeof(int), 4 * n);
  fclose(f);
  for (int k = 0; k < n; ++k) {
    for (int c = 0; c < 3; ++c) t->vnodes[k].p[c] = pos[3 * k + c];
    t->connections[k].forward = iv[k];
    t->connections[k].reverse = iv[n + k];
    t->status[k].status = (node_status_t)iv[2 * n + k];
    t->status[k].pin_wall = (boundary_faces)iv[3 * n + k];
  }
  t->next_free = 0;
  t->total_free = 0;
  if (refh_set_box(t, prm + 12, prm + 15, walls, bimg) != 0) {
    fprintf(stderr, "unknown boundary %s\n", bimg);
    return 2;
  }
  global_use_BH = hdr[2];
  global_BH_resolution = prm[0];
  const double dt = prm[1], rec_dist = prm[2], rec_angle = prm[3];
  const double dl_min = prm[4], dl_max = prm[5];
  VORTEX_WIDTH = prm[6];
  global_alpha = prm[7];
  global_alpha_p = prm[8];
  global_use_mutual_friction = 1;
  global_hyperfriction = 1;
  global_dl_max = dl_max;
  global_num_threads = 4;
  const char *vname = "external_v";
  refh_set_flow(0, "simple", 1, &vname, prm + 9);   /* vn = prm[9..11] */
  refh_set_flow(1, "no flow", 0, NULL, NULL);
  refh_set_flow(2, "no flow", 0, NULL, NULL);

  /* before the loop, as main does (src/main.c:77-85) */
  enforce_boundaries(t);
  update_tangents_normals(t);
  remesh(t, dl_min, dl_max);
  eliminate_small_loops(t, global_small_loop_cutoff);
  update_tangle(t, 0);
  double time = 0;
  int recs = 0;
  /* the loop body (src/main.c:96-118) */
  for (int k = 0; k < steps; ++k) {
    recs += reconnect(t, time, rec_dist, rec_angle);
    eliminate_small_loops(t, global_small_loop_cutoff);
    update_tangle(t, time);
    rk4_step(t, time, dt);
    update_tangents_normals(t);
    remesh(t, dl_min, dl_max);
    eliminate_small_loops(t, global_small_loop_cutoff);
    enforce_boundaries(t);
    time += dt;
  }
  FILE *o = fopen(argv[2], "wb");
  if (!o) {
    perror(argv[2]);
    return 2;
  }
  const int N = (int)t->N;
  fwrite(&N, sizeof(int), 1, o);
  fwrite(&recs, sizeof(int), 1, o);
  for (int k = 0; k < N; ++k) fwrite(t->vnodes[k].p, sizeof(double), 3, o);
  for (int k = 0; k < N; ++k) fwrite(&t->connections[k].forward, sizeof(int), 1, o);
  for (int k = 0; k < N; ++k) fwrite(&t->connections[k].reverse, sizeof(int), 1, o);
  for (int k = 0; k < N; ++k) {
    int s = (int)t->status[k].status;
    fwrite(&s, sizeof(int), 1, o);
  }
  fclose(o);
  printf("steps %d reconnections %d nodes %d\n", steps, recs, N);
  return 0;
}
