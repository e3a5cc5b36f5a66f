/*
 * ov_oracle.c - CPU restatement of OpenVort's velocity + Barnes-Hut + RK4
 * path.  TEST INFRASTRUCTURE ONLY (see ov_oracle.h): plain C, written for
 * clarity, not speed.  Every function cites the reference lines it restates
 * (paths relative to the OpenVort checkout).  The reference's quirks are
 * reproduced on purpose, because the product must match the reference:
 *   - RK4 stage 4 advances by dt/2 (src/vortex_dynamics.c:89) unless
 *     rk4_classic is set;
 *   - the Barnes-Hut "quadrupole" terms keep the reference's formulas
 *     (src/octree.c:310-326 with mat3_vmul of src/vec3_maths.c:398-403);
 *   - the Barnes-Hut opening test uses a once-wrapped distance to the cell's
 *     centre of mass while the expansion uses the unwrapped one
 *     (src/octree.c:286,304);
 *   - nodes outside a child box (strict inequalities) are dropped from the
 *     subtree (src/vec3_maths.c:67-77, src/octree.c:118-127).
 */
#include "ov_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#ifndef M_E
#define M_E 2.7182818284590452354
#endif

typedef struct { double x[3]; } v3;

static v3 mk(double a, double b, double c) { v3 r = {{a, b, c}}; return r; }
static v3 at(const double *p, int k) { return mk(p[3 * k], p[3 * k + 1], p[3 * k + 2]); }
static v3 add(v3 a, v3 b) { return mk(a.x[0] + b.x[0], a.x[1] + b.x[1], a.x[2] + b.x[2]); }
static v3 sub(v3 a, v3 b) { return mk(a.x[0] - b.x[0], a.x[1] - b.x[1], a.x[2] - b.x[2]); }
static v3 scl(v3 a, double s) { return mk(a.x[0] * s, a.x[1] * s, a.x[2] * s); }
/* sequential dot product, as vec3_dot (src/vec3_maths.c:286-292) */
static double dot(v3 a, v3 b) {
  double o = 0;
  for (int k = 0; k < 3; ++k) o += a.x[k] * b.x[k];
  return o;
}
static double norm(v3 a) { return sqrt(dot(a, a)); }
static v3 cross(v3 u, v3 v) {
  return mk(u.x[1] * v.x[2] - u.x[2] * v.x[1], u.x[2] * v.x[0] - u.x[0] * v.x[2],
            u.x[0] * v.x[1] - u.x[1] * v.x[0]);
}

/* inward normals of the box faces (src/vec3_maths.c:55-62) */
static const double face_normal[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0},
                                         {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};

static double box_len(const ovo_tangle *t, int c) { return t->hi[c] - t->lo[c]; }

/* Second endpoint moved by at most one box length per periodic axis so that
 * the segment is short (seg_pwrap, src/vec3_maths.c:105-138).  Returns the
 * moved r2. */
static v3 pwrap(const ovo_tangle *t, v3 r1, v3 r2) {
  for (int c = 0; c < 3; ++c) {
    if (t->wall[2 * c] != OVO_WALL_PERIODIC) continue;
    double L = box_len(t, c);
    double d = r2.x[c] - r1.x[c];
    if (d > L / 2)
      r2.x[c] -= L;
    else if (d < -L / 2)
      r2.x[c] += L;
  }
  return r2;
}

/* reflection of a position in a wall plane (mirror_shift, src/vec3_maths.c:204-258) */
static v3 mirror_pos(const ovo_tangle *t, v3 v, int face) {
  int c = face / 2;
  double w = (face % 2 == 0) ? t->lo[c] : t->hi[c];
  v.x[c] = 2 * w - v.x[c];
  return v;
}

/* reflection of a direction (mirror_dir_reflect, src/vec3_maths.c:260-273) */
static v3 mirror_dir(v3 v, int face) {
  v3 n = mk(face_normal[face][0], face_normal[face][1], face_normal[face][2]);
  double nc = dot(v, n);
  return add(v, scl(n, -2 * nc));
}

/* ---------------------------------------------------------------------- */
/* link walking (step_node, arc_length: src/tangle.c:165-243)              */

static int is_pinned(const ovo_tangle *t, int k) {
  return t->status[k] == OVO_PINNED || t->status[k] == OVO_PINNED_SLIP;
}

static v3 step_node(const ovo_tangle *t, int i, int where) {
  if (where == 0) return at(t->pos, i);
  if (!is_pinned(t, i)) {
    return where > 0 ? step_node(t, t->fwd[i], where - 1)
                     : step_node(t, t->rev[i], where + 1);
  }
  /* pinned: walking off the wall end continues on the mirror image */
  if (where > 0) {
    if (t->fwd[i] >= 0) return step_node(t, t->fwd[i], where - 1);
  } else {
    if (t->rev[i] >= 0) return step_node(t, t->rev[i], where + 1);
  }
  return mirror_pos(t, step_node(t, i, -where), t->pin_wall[i]);
}

static double arc_length(const ovo_tangle *t, const double *dxi, int k, int dist) {
  if (dist == 0) return 0;
  if (is_pinned(t, k)) {
    if (dist > 0 && t->fwd[k] < 0) return arc_length(t, dxi, k, -dist);
    if (dist < 0 && t->rev[k] < 0) return arc_length(t, dxi, k, -dist);
  }
  if (dist > 0) return dxi[k] + arc_length(t, dxi, t->fwd[k], dist - 1);
  return arc_length(t, dxi, t->rev[k], 1) + arc_length(t, dxi, t->rev[k], dist + 1);
}

/* ---------------------------------------------------------------------- */
/* tangents and normals                                                    */

/* Derivative weights at x=0 of the Lagrange interpolant through x=0 and the
 * four offsets x[0..3]: w1 = d/dx, w2 = d2/dx2 of each basis polynomial of
 * the four off-centre points.  Equivalent to the 4-point non-uniform
 * stencils of src/tangle.c:312-344 and :434-470 (derived in 4point.wxmx). */
static void lagrange_weights(const double x[4], double w1[4], double w2[4]) {
  for (int j = 0; j < 4; ++j) {
    double o[3];
    int m = 0;
    for (int k = 0; k < 4; ++k)
      if (k != j) o[m++] = x[k];
    double den = x[j] * (x[j] - o[0]) * (x[j] - o[1]) * (x[j] - o[2]);
    w1[j] = -(o[0] * o[1] * o[2]) / den;
    w2[j] = 2 * (o[0] * o[1] + o[0] * o[2] + o[1] * o[2]) / den;
  }
}

/* s' and s'' of node k from the four stencil points p[j] at arc offsets x[j]:
 * s^(n)(0) = sum_j w_n[j] (p_j - p_0). */
static void stencil4(const ovo_tangle *t, v3 s0, const v3 p[4], const double x[4],
                     v3 *tan, v3 *nrm) {
  double w1[4], w2[4];
  lagrange_weights(x, w1, w2);
  v3 a = mk(0, 0, 0), b = mk(0, 0, 0);
  for (int j = 0; j < 4; ++j) {
    v3 d = sub(pwrap(t, p[j], s0), p[j]); /* s0 - p_j, wrapped */
    a = add(a, scl(d, -w1[j]));
    b = add(b, scl(d, -w2[j]));
  }
  *tan = a;
  *nrm = b;
}

/* one-sided stencil at a pinned node (src/tangle.c:275-364) */
static void tn_pinned(const ovo_tangle *t, const double *dxi, int k, v3 *tan, v3 *nrm) {
  v3 s0 = at(t->pos, k), p[4];
  double x[4];
  /* reference tests forward > 0 (so a forward link to slot 0 walks backwards) */
  int dir = t->fwd[k] > 0 ? 1 : -1;
  for (int j = 0; j < 4; ++j) {
    x[j] = dir * arc_length(t, dxi, k, dir * (j + 1));
    p[j] = step_node(t, k, dir * (j + 1));
  }
  stencil4(t, s0, p, x, tan, nrm);
}

/* free node next to a pinned one: Hermite-type stencil from the neighbours'
 * positions and tangents (src/tangle.c:366-430) */
static void tn_near_pin(const ovo_tangle *t, const double *dxi, const double *tangents,
                        int k, v3 *tan, v3 *nrm) {
  v3 s0 = at(t->pos, k);
  v3 s1 = step_node(t, k, 1), sm1 = step_node(t, k, -1);
  v3 ds1 = sub(pwrap(t, s1, s0), s1);    /* s0 - s1 */
  v3 dsm1 = sub(pwrap(t, sm1, s0), sm1); /* s0 - s_-1 */
  double a = arc_length(t, dxi, k, 1), b = -arc_length(t, dxi, k, -1);
  v3 t1 = at(tangents, t->fwd[k]), tm1 = at(tangents, t->rev[k]);
  double h = a - b, h2 = h * h, h3 = h2 * h;
  double ct1 = -b * b / h2, ctm1 = -a * a / h2;
  double cs1 = 2 * b * b * (b - 2 * a) / (a * h3);
  double csm1 = 2 * a * a * (2 * b - a) / (b * h3);
  double cn1 = 2 * b * (8 * a * a - a * b - b * b) / (a * a * h3);
  double cnm1 = 2 * a * (a * a + a * b - 8 * b * b) / (b * b * h3);
  double cnt1 = 2 * b * (2 * a + b) / (a * h2);
  double cntm1 = 2 * a * (a + 2 * b) / (b * h2);
  *tan = add(add(scl(t1, ct1), scl(tm1, ctm1)), add(scl(ds1, cs1), scl(dsm1, csm1)));
  *nrm = add(add(scl(t1, cnt1), scl(tm1, cntm1)), add(scl(ds1, cn1), scl(dsm1, cnm1)));
}

static void tn_free(const ovo_tangle *t, const double *dxi, int k, v3 *tan, v3 *nrm) {
  v3 s0 = at(t->pos, k), p[4];
  double x[4];
  static const int off[4] = {2, 1, -1, -2};
  for (int j = 0; j < 4; ++j) {
    p[j] = step_node(t, k, off[j]);
    x[j] = off[j] > 0 ? arc_length(t, dxi, k, off[j]) : -arc_length(t, dxi, k, off[j]);
  }
  stencil4(t, s0, p, x, tan, nrm);
}

void ovo_tangents_normals(const ovo_tangle *t, double *dxi, double *tangents,
                          double *normals) {
  /* dxi: length of the forward segment (initialize_dxi, src/tangle.c:704-721) */
  for (int k = 0; k < t->n; ++k) {
    if (t->status[k] == OVO_EMPTY) continue;
    v3 s0 = at(t->pos, k), s1 = step_node(t, k, 1);
    dxi[k] = norm(sub(s0, pwrap(t, s0, s1)));
  }
  /* pass 1: pinned nodes; pass 2: ordinary nodes; pass 3: nodes next to a
   * pinned node, which use their neighbours' tangents (src/tangle.c:366-372) */
  for (int pass = 0; pass < 3; ++pass) {
    for (int k = 0; k < t->n; ++k) {
      int st = t->status[k];
      if (st == OVO_EMPTY) continue;
      v3 tan, nrm;
      int near_pin = st != OVO_PINNED &&
                     ((t->fwd[k] >= 0 && t->status[t->fwd[k]] == OVO_PINNED) ||
                      (t->rev[k] >= 0 && t->status[t->rev[k]] == OVO_PINNED));
      if (st == OVO_PINNED) {
        if (pass != 0) continue;
        tn_pinned(t, dxi, k, &tan, &nrm);
      } else if (near_pin) {
        if (pass != 2) continue;
        tn_near_pin(t, dxi, tangents, k, &tan, &nrm);
      } else {
        if (pass != 1) continue;
        tn_free(t, dxi, k, &tan, &nrm);
      }
      for (int c = 0; c < 3; ++c) {
        tangents[3 * k + c] = tan.x[c];
        normals[3 * k + c] = nrm.x[c];
      }
    }
  }
}

/* ---------------------------------------------------------------------- */
/* external flows (src/external_velocity.c:176-511)                        */

static v3 flow_eval(const ovo_flow *f, v3 w, double time) {
  const double *s = f->s;
  v3 r = mk(0, 0, 0);
  switch (f->kind) {
  case OVO_FLOW_NONE:
    break;
  case OVO_FLOW_SIMPLE:
    r = mk(f->v[0][0], f->v[0][1], f->v[0][2]);
    break;
  case OVO_FLOW_SPHERICAL:
  case OVO_FLOW_SPHERICAL_SIMPLE: {
    /* s[0] strength, s[1] cutoff (src/external_velocity.c:197-223) */
    double rr = norm(w);
    double attn = (s[1] / rr) * (s[1] / rr);
    if (!(rr < 1e-8 || attn > 100)) {
      double fac = exp(-attn);
      r = scl(w, 1 / norm(w));
      r = scl(r, s[0] / (4 * M_PI * rr * rr) * fac);
    }
    /* the reference's combined flow never writes its output (its
     * get_v_simple returns 1, read as an error at :235-237); this restatement
     * returns the evident intent, spherical + simple */
    if (f->kind == OVO_FLOW_SPHERICAL_SIMPLE)
      r = add(r, mk(f->v[0][0], f->v[0][1], f->v[0][2]));
    break;
  }
  case OVO_FLOW_CYLINDRICAL: { /* s[0] strength, s[1] cutoff (:243-270) */
    double rr = sqrt(w.x[0] * w.x[0] + w.x[1] * w.x[1]);
    double attn = (s[1] / rr) * (s[1] / rr);
    if (!(rr < 1e-8 || attn > 100)) {
      double fac = exp(-attn);
      r = mk(w.x[0], w.x[1], 0);
      r = scl(r, 1 / norm(r));
      r = scl(r, s[0] / (2 * M_PI * rr) * fac);
    }
    break;
  }
  case OVO_FLOW_OSCILLATING: { /* s[0] strength, s[1] frequency, v[0] wave, v[1] pol (:272-294) */
    v3 k = mk(f->v[0][0], f->v[0][1], f->v[0][2]);
    double X = cos(2 * M_PI * dot(k, w));
    double T = sin(2 * M_PI * s[1] * time);
    r = scl(mk(f->v[1][0], f->v[1][1], f->v[1][2]), s[0] * X * T);
    break;
  }
  case OVO_FLOW_OSCILLATING_SLIT: { /* s[0] strength (unused), s[1] freq, s[2] cutoff (:296-322) */
    double x = w.x[0], z = w.x[2];
    double rr = sqrt(x * x + z * z);
    v3 dir = mk(x / rr, 0, z / rr);
    double attn = exp(-s[2] * s[2] / rr / rr);
    double osc = cos(2 * M_PI * s[1] * time);
    r = scl(dir, osc * attn);
    break;
  }
  case OVO_FLOW_COSCOS: /* s[0] k, s[1] v0, s[2] l (:324-344) */
    r.x[2] = s[1] * (1 + cos(s[0] * w.x[0]) * cos(s[0] * w.x[1]) * exp(-w.x[2] / s[2]));
    break;
  case OVO_FLOW_COSCOS_DIVFREE: { /* (:347-370) */
    double k = s[0], v0 = s[1], l = s[2], x = w.x[0], y = w.x[1], z = w.x[2];
    r.x[0] = v0 / 2 / l / k * sin(k * x) * cos(k * y) * exp(-z / l);
    r.x[1] = v0 / 2 / l / k * cos(k * x) * sin(k * y) * exp(-z / l);
    r.x[2] = v0 * (1 + cos(k * x) * cos(k * y) * exp(-z / l));
    break;
  }
  case OVO_FLOW_COS_DIVFREE: { /* (:372-394) */
    double k = s[0], v0 = s[1], l = s[2], x = w.x[0], z = w.x[2];
    r.x[0] = v0 / l / k * sin(k * x) * exp(-z / l);
    r.x[2] = v0 * (1 + cos(k * x) * exp(-z / l));
    break;
  }
  case OVO_FLOW_SIMPLE_SHEAR: /* s[0] rate, s[1] v0 (:396-413) */
    r.x[2] = s[1] + s[0] * w.x[0];
    break;
  case OVO_FLOW_ROTOSC:
  case OVO_FLOW_ROTOSC_BOUNDARY: /* s[0] freq, s[1] amp (:415-433); the table
                                    maps "rotosc-boundary" to the same function */
    r = scl(cross(mk(0, 0, 1), w), s[1] * cos(2 * M_PI * s[0] * time));
    break;
  case OVO_FLOW_DG: /* s[0] rot, s[1] vz (:438-457) */
    r = scl(cross(mk(0, 0, 1), w), s[0]);
    r.x[2] += s[1];
    break;
  case OVO_FLOW_CONST_ACCEL: /* s[0] accel (:483-495) */
    r = mk(s[0] * time, 0, 0);
    break;
  case OVO_FLOW_PARABOLIC: /* s[0] H, s[1] amp (:497-511) */
    r = mk(s[1] * w.x[2] * (s[0] - w.x[2]), 0, 0);
    break;
  default:
    break;
  }
  return r;
}

/* ---------------------------------------------------------------------- */
/* Biot-Savart                                                             */

/* straight segment r1->r2 at point r (segment_field1, src/tangle.c:486-514) */
static v3 segment_vel(double kappa, v3 r1, v3 r2, v3 r) {
  v3 R = sub(r1, r), Rp = sub(r2, r);
  double lR = norm(R), lRp = norm(Rp);
  double denom = lR * lRp * (lR * lRp + dot(R, Rp));
  double f = kappa / 4 / M_PI;
  if (lR < 1e-8 || lRp < 1e-8) return mk(0, 0, 0);
  if (fabs(dot(R, Rp) / norm(R) / norm(Rp) - 1) < 1e-8) return mk(0, 0, 0);
  return scl(cross(R, Rp), f * (lR + lRp) / denom);
}

/* segment starting at node m (segment_field, src/tangle.c:519-528) */
static v3 node_segment_vel(const ovo_tangle *t, double kappa, int m, v3 r) {
  int nx = t->fwd[m];
  if (nx == -1) return mk(0, 0, 0);
  v3 r1 = at(t->pos, m);
  return segment_vel(kappa, r1, pwrap(t, r1, at(t->pos, nx)), r);
}

/* sum over the given nodes' segments with the skip rule
 * (calculate_vs_shift, src/tangle.c:553-576) */
static v3 segment_sum(const ovo_tangle *t, double kappa, v3 r, int skip, const int *ids,
                      int nids, v3 vs) {
  int n = ids ? nids : t->n;
  for (int m = 0; m < n; ++m) {
    int k = ids ? ids[m] : m;
    if (t->fwd[k] == -1 || skip == k || skip == t->fwd[k]) continue;
    vs = add(vs, node_segment_vel(t, kappa, k, r));
  }
  return vs;
}

/* image position (shifted, src/tangle.c:39-79) */
static v3 image_point(const ovo_tangle *t, const int *img, v3 r) {
  v3 rs = r;
  for (int c = 0; c < 3; ++c) rs.x[c] -= box_len(t, c) * img[c];
  int face = img[3];
  if (face >= 0) {
    int c = face / 2;
    double w = (face % 2 == 0) ? t->lo[c] : t->hi[c];
    rs.x[c] = 2 * w - r.x[c];
  }
  return rs;
}

/* ---------------------------------------------------------------------- */
/* Barnes-Hut octree (src/octree.c)                                        */

typedef struct cell {
  double lo[3], hi[3];
  int n, cap;
  int *ids;
  double com[3], gam[3], M[3][3];
  struct cell *ch[8];
  int nch; /* 0 when not split */
} cell;

static double box_max(const double lo[3], const double hi[3]) {
  double L[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
  if (L[0] > L[1]) return L[0] > L[2] ? L[0] : L[2];
  return L[1] > L[2] ? L[1] : L[2];
}
static double box_min(const double lo[3], const double hi[3]) {
  double L[3] = {hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]};
  if (L[0] < L[1]) return L[0] < L[2] ? L[0] : L[2];
  return L[1] < L[2] ? L[1] : L[2];
}

/* Child box k of a parent box, with the reference's exact arithmetic and
 * child numbering (make_child_box, src/octree.c:158-235):
 *   k : 0 BLF  1 BLB  2 BRF  3 BRB  4 TLF  5 TLB  6 TRF  7 TRB
 *   x : hi   lo   hi   lo   hi   lo   hi   lo
 *   y : lo   lo   hi   hi   lo   lo   hi   hi
 *   z : lo   lo   lo   lo   hi   hi   hi   hi   (quadtree: z not split) */
static void child_box(const double plo[3], const double phi[3], int k, int quad,
                      double lo[3], double hi[3]) {
  double c[3], L[3];
  for (int a = 0; a < 3; ++a) {
    c[a] = (plo[a] + phi[a]) * 0.5;
    L[a] = phi[a] - plo[a];
  }
  /* "shift" cases move a corner box by half a length along one axis */
  switch (k) {
  case 0: memcpy(lo, plo, 24); memcpy(hi, c, 24); lo[0] += L[0] / 2; hi[0] += L[0] / 2; break;
  case 1: memcpy(lo, plo, 24); memcpy(hi, c, 24); break;
  case 2: memcpy(lo, c, 24); memcpy(hi, phi, 24); lo[2] -= L[2] / 2; hi[2] -= L[2] / 2; break;
  case 3: memcpy(lo, plo, 24); memcpy(hi, c, 24); lo[1] += L[1] / 2; hi[1] += L[1] / 2; break;
  case 4: memcpy(lo, c, 24); memcpy(hi, phi, 24); lo[1] -= L[1] / 2; hi[1] -= L[1] / 2; break;
  case 5: memcpy(lo, plo, 24); memcpy(hi, c, 24); lo[2] += L[2] / 2; hi[2] += L[2] / 2; break;
  case 6: memcpy(lo, c, 24); memcpy(hi, phi, 24); break;
  default: memcpy(lo, c, 24); memcpy(hi, phi, 24); lo[0] -= L[0] / 2; hi[0] -= L[0] / 2; break;
  }
  if (quad) hi[2] = phi[2];
}

static int strictly_inside(const double lo[3], const double hi[3], v3 p) {
  return p.x[0] > lo[0] && p.x[0] < hi[0] && p.x[1] > lo[1] && p.x[1] < hi[1] &&
         p.x[2] > lo[2] && p.x[2] < hi[2];
}

static cell *cell_new(int cap) {
  cell *c = (cell *)calloc(1, sizeof(cell));
  c->cap = cap > 0 ? cap : 1;
  c->ids = (int *)malloc(sizeof(int) * c->cap);
  return c;
}

static void cell_push(cell *c, int id) {
  if (c->n == c->cap) {
    c->cap *= 2;
    c->ids = (int *)realloc(c->ids, sizeof(int) * c->cap);
  }
  c->ids[c->n++] = id;
}

static void cell_free(cell *c) {
  if (!c) return;
  for (int k = 0; k < c->nch; ++k) cell_free(c->ch[k]);
  free(c->ids);
  free(c);
}

/* node-list moments (octree_update_means, src/octree.c:237-272) */
static void cell_moments(const ovo_tangle *t, cell *c) {
  if (c->n == 0) return;
  v3 s = mk(0, 0, 0);
  for (int k = 0; k < c->n; ++k) s = add(s, at(t->pos, c->ids[k]));
  s = scl(s, 1.0 / c->n);
  v3 g = mk(0, 0, 0);
  double M[3][3] = {{0}};
  for (int k = 0; k < c->n; ++k) {
    int id = c->ids[k];
    if (t->fwd[id] < 0) continue;
    v3 p = at(t->pos, id);
    v3 ds = sub(pwrap(t, p, at(t->pos, t->fwd[id])), p);
    g = add(g, ds);
    v3 loc = sub(p, s);
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) M[i][j] += ds.x[i] * loc.x[j];
  }
  memcpy(c->com, s.x, 24);
  memcpy(c->gam, g.x, 24);
  memcpy(c->M, M, sizeof(M));
}

/* recursive split (octree_inner_sort, src/octree.c:99-136) */
static void cell_split(const ovo_tangle *t, const ovo_params *p, cell *c) {
  if (c->n <= 1) return;
  if (box_min(c->lo, c->hi) < p->bh_grain * p->dl_max) return;
  int nch = p->bh_quadtree ? 4 : 8;
  int cap = c->cap / 8 > 0 ? c->cap / 8 : 8;
  c->nch = nch;
  for (int k = 0; k < nch; ++k) {
    c->ch[k] = cell_new(cap);
    child_box(c->lo, c->hi, k, p->bh_quadtree, c->ch[k]->lo, c->ch[k]->hi);
  }
  for (int m = 0; m < c->n; ++m) {
    v3 q = at(t->pos, c->ids[m]);
    for (int k = 0; k < nch; ++k) {
      if (strictly_inside(c->ch[k]->lo, c->ch[k]->hi, q)) {
        cell_push(c->ch[k], c->ids[m]);
        break;
      }
    }
  }
  for (int k = 0; k < nch; ++k) cell_split(t, p, c->ch[k]);
}

static void cell_all_moments(const ovo_tangle *t, cell *c) {
  cell_moments(t, c);
  for (int k = 0; k < c->nch; ++k) cell_all_moments(t, c->ch[k]);
}

/* octree_build (src/octree.c:79-96) */
static cell *tree_build(const ovo_tangle *t, const ovo_params *p) {
  cell *root = cell_new(t->n);
  for (int k = 0; k < t->n; ++k)
    if (t->status[k] != OVO_EMPTY) cell_push(root, k);
  memcpy(root->lo, t->lo, 24);
  memcpy(root->hi, t->hi, 24);
  cell_split(t, p, root);
  cell_all_moments(t, root);
  return root;
}

/* Barnes-Hut velocity at r (octree_get_vs, src/octree.c:275-343) */
static v3 tree_vel(const ovo_tangle *t, const ovo_params *p, const cell *c, v3 r, int skip) {
  if (!c || c->n == 0) return mk(0, 0, 0);
  double Lm = box_max(c->lo, c->hi), Lmin = box_min(c->lo, c->hi);
  v3 com = mk(c->com[0], c->com[1], c->com[2]);
  double d = norm(sub(r, pwrap(t, r, com)));
  if (c->n == 1 || Lmin < p->bh_grain) return segment_sum(t, p->kappa, r, skip, c->ids, c->n, mk(0, 0, 0));
  if (d > 0 && Lm / d < p->bh_theta) {
    v3 R = sub(r, com);
    double Rm = norm(R);
    v3 res = scl(cross(mk(c->gam[0], c->gam[1], c->gam[2]), R), 1 / Rm / Rm / Rm);
    /* the reference's Levi-Civita loop only ever sets component 0 */
    res = add(res, scl(mk(c->M[2][1], 0, 0), 1 / Rm / Rm / Rm));
    /* the reference's matrix-vector product keeps only the j=2 column */
    v3 mv = mk(c->M[0][2] * R.x[2], c->M[1][2] * R.x[2], c->M[2][2] * R.x[2]);
    res = add(res, scl(cross(mv, R), 1 / Rm / Rm / Rm / Rm / Rm));
    return scl(res, p->kappa / 4 / M_PI);
  }
  v3 tot = mk(0, 0, 0);
  for (int k = 0; k < c->nch; ++k) tot = add(tot, tree_vel(t, p, c->ch[k], r, skip));
  return tot;
}

/* ---------------------------------------------------------------------- */
/* per-node velocity (update_velocity, src/tangle.c:583-684)               */

static void node_velocity(const ovo_tangle *t, const ovo_params *p, const cell *tree,
                          double time, const double *tangents, const double *normals,
                          int k, double *vels, double *vs_out) {
  int st = t->status[k];
  if (st == OVO_EMPTY) return;
  v3 r = at(t->pos, k);
  if (st == OVO_PINNED) {
    v3 vb = flow_eval(&p->vb, r, time);
    for (int c = 0; c < 3; ++c) {
      vs_out[3 * k + c] = 0;
      vels[3 * k + c] = vb.x[c];
    }
    return;
  }
  v3 tan = at(tangents, k), nrm = at(normals, k);
  /* local induction term (lia_velocity, src/tangle.c:530-551) */
  v3 nx = step_node(t, k, 1), pv = step_node(t, k, -1);
  double l_next = norm(sub(r, pwrap(t, r, nx)));
  double l_prev = norm(sub(pv, pwrap(t, pv, r)));
  double f = p->kappa * log(2 * sqrt(l_next * l_prev) / sqrt(sqrt(M_E)) / p->core_a) / 4 / M_PI;
  v3 lia = scl(cross(tan, nrm), f);
  v3 vs = add(lia, flow_eval(&p->vs, r, time));
  if (!p->lia_only) {
    if (p->use_bh && tree)
      vs = add(vs, tree_vel(t, p, tree, r, k));
    else
      vs = segment_sum(t, p->kappa, r, k, NULL, 0, vs); /* accumulates onto vs as :612-619 */
    v3 vimg = mk(0, 0, 0);
    for (int j = 0; j < t->n_img; ++j) {
      const int *img = t->img + 4 * j;
      v3 rs = image_point(t, img, r);
      v3 vj = (p->use_bh && tree) ? tree_vel(t, p, tree, rs, -1)
                                  : segment_sum(t, p->kappa, rs, -1, NULL, 0, mk(0, 0, 0));
      if (img[3] > -1) vj = mirror_dir(vj, img[3]);
      vimg = add(vimg, vj);
    }
    vs = add(vs, vimg);
  }
  v3 v = vs;
  if (p->hyperfriction) {
    if (norm(nrm) > p->max_curv_scale / p->dl_max)
      v = add(v, scl(cross(tan, lia), -p->hyperalpha));
  }
  if (p->use_mf) {
    v3 dv = sub(flow_eval(&p->vn, r, time), vs);
    v = add(v, scl(cross(tan, dv), p->alpha));
    v = add(v, scl(cross(tan, cross(tan, dv)), -p->alpha_p));
  }
  if (st == OVO_PINNED_SLIP) {
    int w = t->pin_wall[k];
    v3 n = mk(face_normal[w][0], face_normal[w][1], face_normal[w][2]);
    v = sub(v, scl(n, dot(n, v)));
  }
  for (int c = 0; c < 3; ++c) {
    vs_out[3 * k + c] = vs.x[c];
    vels[3 * k + c] = v.x[c];
  }
}

void ovo_velocities(const ovo_tangle *t, const ovo_params *p, double time,
                    const double *tangents, const double *normals, double *vels,
                    double *vs) {
  cell *tree = p->use_bh ? tree_build(t, p) : NULL;
#pragma omp parallel for schedule(dynamic, 16)
  for (int k = 0; k < t->n; ++k)
    node_velocity(t, p, tree, time, tangents, normals, k, vels, vs);
  cell_free(tree);
}

void ovo_segments_at(const ovo_tangle *t, const ovo_params *p, int npts,
                     const double *pts, const int *skip, double *out) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < npts; ++i) {
    v3 v = segment_sum(t, p->kappa, at(pts, i), skip ? skip[i] : -1, NULL, 0, mk(0, 0, 0));
    for (int c = 0; c < 3; ++c) out[3 * i + c] = v.x[c];
  }
}

void ovo_bh_at(const ovo_tangle *t, const ovo_params *p, int npts, const double *pts,
               const int *skip, double *out) {
  cell *tree = tree_build(t, p);
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < npts; ++i) {
    v3 v = tree_vel(t, p, tree, at(pts, i), skip ? skip[i] : -1);
    for (int c = 0; c < 3; ++c) out[3 * i + c] = v.x[c];
  }
  cell_free(tree);
}

void ovo_update_tangle(const ovo_tangle *t, const ovo_params *p, double time,
                       double *dxi, double *tangents, double *normals,
                       double *vels, double *vs) {
  ovo_tangents_normals(t, dxi, tangents, normals);
  ovo_velocities(t, p, time, tangents, normals, vels, vs);
}

/* ---------------------------------------------------------------------- */
/* RK4 (rk4_step2, src/vortex_dynamics.c:58-117)                          */

void ovo_rk4_step(const ovo_tangle *t, const ovo_params *p, double time, double dt,
                  double *pos, const double *vels_k1) {
  int n = t->n;
  size_t sz = sizeof(double) * 3 * (size_t)n;
  double *stage = (double *)malloc(sz), *dxi = (double *)malloc(sizeof(double) * n);
  double *tg = (double *)malloc(sz), *nm = (double *)malloc(sz), *vs = (double *)malloc(sz);
  double *k[3];
  for (int s = 0; s < 3; ++s) k[s] = (double *)calloc((size_t)3 * n, sizeof(double));
  ovo_tangle ts = *t;
  ts.pos = stage;
  const double h[3] = {dt / 2, dt / 2, p->rk4_classic ? dt : dt / 2};
  const double tt[3] = {time + dt / 2, time + dt / 2, time + dt};
  memcpy(stage, pos, sz);
  for (int s = 0; s < 3; ++s) {
    const double *prev = s == 0 ? vels_k1 : k[s - 1];
    for (int i = 0; i < n; ++i) {
      if (t->status[i] == OVO_EMPTY) continue;
      for (int c = 0; c < 3; ++c) stage[3 * i + c] = pos[3 * i + c] + prev[3 * i + c] * h[s];
    }
    ovo_tangents_normals(&ts, dxi, tg, nm);
    ovo_velocities(&ts, p, tt[s], tg, nm, k[s], vs);
  }
  for (int i = 0; i < n; ++i) {
    if (t->status[i] == OVO_EMPTY) continue;
    for (int c = 0; c < 3; ++c) {
      double mv = vels_k1[3 * i + c] * (dt / 6);
      mv += k[0][3 * i + c] * (dt / 3);
      mv += k[1][3 * i + c] * (dt / 3);
      mv += k[2][3 * i + c] * (dt / 6);
      pos[3 * i + c] += mv;
    }
  }
  for (int s = 0; s < 3; ++s) free(k[s]);
  free(stage); free(dxi); free(tg); free(nm); free(vs);
}
