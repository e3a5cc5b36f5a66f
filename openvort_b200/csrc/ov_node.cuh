// ov_node.cuh - per-node geometry and velocity assembly as device
// functions: the segment length to the next node, the 4-point tangent and
// normal stencils, and the epilogue of update_velocity, for the per-node
// kernels (ov_geom.cu) and any kernel that must give their bits.
#pragma once

#include "ov_internal.h"
#include "ov_links.cuh"

namespace {

// s' and s'' at x=0 from four points p_j at arc offsets x_j: weights are the
// first and second derivatives at 0 of the Lagrange basis through {0, x_j}
// (the 4-point non-uniform stencils of src/tangle.c:312-344,434-470).
__device__ void stencil4(const OvParams& P, d3 s0, const d3 p[4], const double x[4],
                         d3& tan, d3& nrm) {
  d3 a = mk3(0, 0, 0), b = mk3(0, 0, 0);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    double o0 = x[(j + 1) & 3], o1 = x[(j + 2) & 3], o2 = x[(j + 3) & 3];
    double den = x[j] * (x[j] - o0) * (x[j] - o1) * (x[j] - o2);
    double w1 = -(o0 * o1 * o2) / den;
    double w2 = 2.0 * (o0 * o1 + o0 * o2 + o1 * o2) / den;
    d3 d = pwrap(P, p[j], s0) - p[j];   // s0 - p_j (wrapped)
    a = a + d * (-w1);
    b = b + d * (-w2);
  }
  tan = a;
  nrm = b;
}

// dxi: distance to the next node after the periodic wrap (arc_length's
// segment lengths, src/tangle.c:165-200 and initialize_dxi)
__device__ __forceinline__ bool dxi_node(const OvParams& P, const Links& L, const double* pos, int k,
                                         double& out) {
  d3 s0 = ld3(pos, k), s1;
  if (!step_node(P, L, pos, k, 1, s1)) return false;
  d3 w = pwrap(P, s0, s1);
  out = norm_ref(s0 - w);
  return true;
}

// a node next to a pinned one (its stencil reads its neighbours' tangents)
__device__ __forceinline__ bool near_pinned(const Links& L, int k) {
  const int2 st = L.st[k], lk = L.lk[k];
  return st.x != OV_PINNED &&
         ((lk.x >= 0 && L.st[lk.x].x == OV_PINNED) || (lk.y >= 0 && L.st[lk.y].x == OV_PINNED));
}

// s' and s'' of node k (update_tangent_normal, src/tangle.c:275-480):
// one-sided stencils at pinned nodes, the neighbours' tangents next to a
// pinned node (read from tan), 4-point stencils elsewhere.  arc(k, dist,
// out) gives the arc length dist links away.  False on a broken link.
template <class Arc>
__device__ bool tangent_node(const OvParams& P, const Links& L, const double* pos, int k, Arc&& arc,
                             const double* tan, d3& t, d3& nn) {
  const int2 st = L.st[k], lk = L.lk[k];
  const d3 s0 = ld3(pos, k);
  bool ok = true;
  if (st.x == OV_PINNED) {
    // one-sided stencil away from the wall (src/tangle.c:275-364); the
    // reference tests forward > 0, so a forward link to slot 0 goes backwards
    int dir = lk.x > 0 ? 1 : -1;
    d3 p[4];
    double x[4];
    for (int j = 0; j < 4 && ok; ++j) {
      double a;
      ok = ok && arc(k, dir * (j + 1), a) && step_node(P, L, pos, k, dir * (j + 1), p[j]);
      x[j] = dir * a;
    }
    if (ok) stencil4(P, s0, p, x, t, nn);
  } else if (near_pinned(L, k)) {
    d3 s1, sm1;
    double a, bm;
    ok = step_node(P, L, pos, k, 1, s1) && step_node(P, L, pos, k, -1, sm1) && arc(k, 1, a) && arc(k, -1, bm);
    if (ok) {
      double b = -bm;
      d3 ds1 = pwrap(P, s1, s0) - s1, dsm1 = pwrap(P, sm1, s0) - sm1;
      d3 t1 = ld3(tan, lk.x), tm1 = ld3(tan, lk.y);
      double h = a - b, h2 = h * h, h3 = h2 * h;
      double ct1 = -b * b / h2, ctm1 = -a * a / h2;
      double cs1 = 2 * b * b * (b - 2 * a) / (a * h3);
      double csm1 = 2 * a * a * (2 * b - a) / (b * h3);
      double cn1 = 2 * b * (8 * a * a - a * b - b * b) / (a * a * h3);
      double cnm1 = 2 * a * (a * a + a * b - 8 * b * b) / (b * b * h3);
      double cnt1 = 2 * b * (2 * a + b) / (a * h2);
      double cntm1 = 2 * a * (a + 2 * b) / (b * h2);
      t = (t1 * ct1 + tm1 * ctm1) + (ds1 * cs1 + dsm1 * csm1);
      nn = (t1 * cnt1 + tm1 * cntm1) + (ds1 * cn1 + dsm1 * cnm1);
    }
  } else {
    const int off[4] = {2, 1, -1, -2};
    d3 p[4];
    double x[4];
    for (int j = 0; j < 4 && ok; ++j) {
      double a;
      ok = ok && arc(k, off[j], a) && step_node(P, L, pos, k, off[j], p[j]);
      x[j] = off[j] > 0 ? a : -a;
    }
    if (ok) stencil4(P, s0, p, x, t, nn);
  }
  return ok;
}

// velocity assembly of a non-EMPTY node (update_velocity, src/tangle.c:
// 583-684) from its tangent tg, normal nm and Biot-Savart sums vnl (the
// tangle) and vim (the images) at time t.  Returns error bits: 1 broken
// link (nothing written), 2 non-finite velocity.
__device__ int epilogue_node(const OvParams& P, const Links& L, double t, const double* pos, int k, d3 tg,
                             d3 nm, d3 vnl, d3 vim, d3& v, d3& vs) {
  const int2 st = L.st[k];
  const d3 r = ld3(pos, k);
  if (st.x == OV_PINNED) {
    vs = mk3(0, 0, 0);
    v = flow_eval(P.vb, r, t);
    return 0;
  }
  // local induction (lia_velocity, src/tangle.c:530-551)
  d3 nx, pv;
  if (!step_node(P, L, pos, k, 1, nx) || !step_node(P, L, pos, k, -1, pv)) return 1;
  double l_next = norm_ref(r - pwrap(P, r, nx));
  double l_prev = norm_ref(pv - pwrap(P, pv, r));
  double f = P.kappa * log(2.0 * sqrt(l_next * l_prev) / sqrt(sqrt(OV_E)) / P.core_a) / 4.0 / OV_PI;
  d3 lia = cross3(tg, nm) * f;
  vs = lia + flow_eval(P.vs, r, t);
  if (!P.lia_only) {
    vs = vs + vnl;
    if (P.n_img > 0) vs = vs + vim;
  }
  v = vs;
  if (P.hyperfriction) {
    if (norm_ref(nm) > P.max_curv / P.dl_max) v = v + cross3(tg, lia) * (-P.hyperalpha);
  }
  if (P.use_mf) {
    d3 dv = flow_eval(P.vn, r, t) - vs;
    v = v + cross3(tg, dv) * P.alpha;
    v = v + cross3(tg, cross3(tg, dv)) * (-P.alpha_p);
  }
  if (st.x == OV_PINNED_SLIP) {
    d3 nw = face_normal(st.y);
    v = v - nw * dot3(nw, v);
  }
  return (isfinite(v.x) && isfinite(v.y) && isfinite(v.z)) ? 0 : 2;
}

}  // namespace
