// ov_adjoint.cu - reverse-mode derivatives of the velocity and of an RK4
// trajectory with fixed topology (ov_adjoint_*, include/openvort_b200.h).
//
// Scope: closed loops of free nodes, open boundaries, no images, direct
// Biot-Savart sum (the forward dynamics of update_velocity,
// src/tangle.c:583-684, and rk4_step, src/vortex_dynamics.c:58-121, with
// reconnection and remeshing off).  The normal-fluid flow (mutual friction)
// and the superfluid flow must be "no flow" or "simple"; the derivative with
// respect to the normal-fluid vector is returned.
//
// Velocity of node k: v_k = F(x_{k-2..k+2}, vnl_k, vn), where F is the local
// part (4-point stencils, local induction, hyperfriction, mutual friction)
// and vnl_k = sum over segments m of B(x_m, x_{m+1}; x_k) the nonlocal sum.
// The vector-Jacobian product g -> x_bar:
//   - local part: forward-mode dual numbers, one thread per (node, input):
//     21 inputs (15 neighbour coordinates, vnl_k, vn), each thread returns
//     g_k . dF/d(input) (k_local_vjp);
//   - nonlocal part: the hand-derived reverse of the segment formula, in two
//     all-pairs passes over shared-memory tiles, one accumulating the
//     targets' and one the segment endpoints' cotangents (k_bs_vjp_*).
// RK4 reverse: positions are checkpointed every `every` steps; the reverse
// sweep recomputes one block of steps from its checkpoint, then runs back
// through it, recomputing each step's stage positions (y1..y3) and taking
// the four stage VJPs.
#include <algorithm>
#include <vector>

#include "ov_internal.h"

namespace {

// ---------------------------------------------------------------- duals
struct Dual {
  double v, d;
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.d}; }
__device__ __forceinline__ Dual operator+(Dual a, double b) { return {a.v + b, a.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
  const double q = a.v / b.v;
  return {q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ Dual operator*(Dual a, double s) { return {a.v * s, a.d * s}; }
__device__ __forceinline__ Dual operator*(double s, Dual a) { return {s * a.v, s * a.d}; }
__device__ __forceinline__ Dual operator/(Dual a, double s) { return {a.v / s, a.d / s}; }
__device__ __forceinline__ Dual dsqrt(Dual a) {
  const double r = sqrt(a.v);
  return {r, a.d / (2.0 * r)};
}
__device__ __forceinline__ Dual dlog(Dual a) { return {log(a.v), a.d / a.v}; }
__device__ __forceinline__ double dval(Dual a) { return a.v; }
__device__ __forceinline__ double dsqrt(double a) { return sqrt(a); }
__device__ __forceinline__ double dlog(double a) { return log(a); }
__device__ __forceinline__ double dval(double a) { return a; }

template <class T>
struct V {
  T x, y, z;
};
template <class T>
__device__ __forceinline__ V<T> operator+(V<T> a, V<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T>
__device__ __forceinline__ V<T> operator-(V<T> a, V<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T, class S>
__device__ __forceinline__ V<T> operator*(V<T> a, S s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T>
__device__ __forceinline__ V<T> vcross(V<T> a, V<T> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// sqrt(x*x + y*y + z*z), summed in this order (norm_ref)
template <class T>
__device__ __forceinline__ T vnorm(V<T> a) { return dsqrt(a.x * a.x + a.y * a.y + a.z * a.z); }

struct LocalP {
  double kappa, core_a, alpha, alpha_p, hyperalpha, curv_thr;
  double vs_flow[3];
  int use_mf, hyperfriction, lia_only;
};

// The local part of a free node's velocity from x[0..4] = x_{k-2..k+2}: the
// 4-point stencils of update_tangent_normal (src/tangle.c:434-470, written
// as Lagrange-basis derivative weights as in k_tangents), local induction,
// superfluid flow, the nonlocal sum vnl, hyperfriction and mutual friction
// (update_velocity, src/tangle.c:597-683), in the order of k_epilogue.
template <class T>
__device__ V<T> local_velocity(const LocalP& L, const V<T> (&x)[5], const V<T>& vnl, const V<T>& vn) {
  const V<T> s0 = x[2];
  const T dm2 = vnorm(x[0] - x[1]), dm1 = vnorm(x[1] - x[2]), d0 = vnorm(x[2] - x[3]),
          d1 = vnorm(x[3] - x[4]);
  const V<T> p[4] = {x[4], x[3], x[1], x[0]};
  const T xo[4] = {d0 + d1, d0, -dm1, -(dm1 + dm2)};
  V<T> tg = s0 * 0.0, nm = s0 * 0.0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const T o0 = xo[(j + 1) & 3], o1 = xo[(j + 2) & 3], o2 = xo[(j + 3) & 3];
    const T den = xo[j] * (xo[j] - o0) * (xo[j] - o1) * (xo[j] - o2);
    const T w1 = -(o0 * o1 * o2) / den;
    const T w2 = 2.0 * (o0 * o1 + o0 * o2 + o1 * o2) / den;
    const V<T> d = s0 - p[j];
    tg = tg + d * (-w1);
    nm = nm + d * (-w2);
  }
  const T f = L.kappa * dlog(2.0 * dsqrt(d0 * dm1) / sqrt(sqrt(OV_E)) / L.core_a) / 4.0 / OV_PI;
  const V<T> lia = vcross(tg, nm) * f;
  V<T> vs = lia + V<T>{s0.x * 0.0 + L.vs_flow[0], s0.y * 0.0 + L.vs_flow[1], s0.z * 0.0 + L.vs_flow[2]};
  if (!L.lia_only) vs = vs + vnl;
  V<T> v = vs;
  if (L.hyperfriction && dval(vnorm(nm)) > L.curv_thr) v = v + vcross(tg, lia) * (-L.hyperalpha);
  if (L.use_mf) {
    const V<T> dv = vn - vs;
    v = v + vcross(tg, dv) * L.alpha;
    v = v + vcross(tg, vcross(tg, dv)) * (-L.alpha_p);
  }
  return v;
}

__device__ __forceinline__ V<Dual> seed3(const double* p, int comp_seed) {
  V<Dual> r;
  r.x = {p[0], comp_seed == 0 ? 1.0 : 0.0};
  r.y = {p[1], comp_seed == 1 ? 1.0 : 0.0};
  r.z = {p[2], comp_seed == 2 ? 1.0 : 0.0};
  return r;
}

constexpr int kLocalInputs = 21;

// One thread per (node k, input i): g_k . dF_k/d(input i), added to x_bar of
// the neighbour it belongs to, written as the cotangent of vnl_k, or added
// to vn_bar.
__global__ void k_local_vjp(LocalP L, const double* __restrict__ pos, const int2* __restrict__ links,
                            const int2* __restrict__ status, const double* __restrict__ vnl,
                            const double* __restrict__ vn, const double* __restrict__ g, double* xbar,
                            double* gnl, double* vnbar, int n) {
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int k = (int)(tid / kLocalInputs), i = (int)(tid % kLocalInputs);
  if (k >= n || status[k].x == OV_EMPTY) return;
  const int f1 = links[k].x, b1 = links[k].y;
  const int ids[5] = {links[b1].y, b1, k, f1, links[f1].x};
  V<Dual> x[5];
#pragma unroll
  for (int a = 0; a < 5; ++a) x[a] = seed3(pos + 3 * (size_t)ids[a], i / 3 == a ? i % 3 : -1);
  const V<Dual> dn = seed3(vnl + 3 * (size_t)k, i >= 15 && i < 18 ? i - 15 : -1);
  const V<Dual> dvn = seed3(vn, i >= 18 ? i - 18 : -1);
  const V<Dual> v = local_velocity(L, x, dn, dvn);
  const double* gk = g + 3 * (size_t)k;
  const double c = gk[0] * v.x.d + gk[1] * v.y.d + gk[2] * v.z.d;
  if (i < 15) atomicAdd(&xbar[3 * (size_t)ids[i / 3] + i % 3], c);
  else if (i < 18) gnl[3 * (size_t)k + (i - 15)] = c;
  else atomicAdd(&vnbar[i - 18], c);
}

// ---------------------------------------------------------------- nonlocal
// Reverse of the segment formula seg_vel64 (the reference's segment_field1,
// src/tangle.c:486-517): v = s (R x R'), s = f4pi (a + b) / (P Q), P = ab,
// Q = P + R.R', a = |R|, b = |R'|, R = r1 - r, R' = r2 - r.  Given g, the
// cotangents of R and R' of g . v; zero where the reference's cut-offs
// return zero.
__device__ __forceinline__ void seg_vjp(double f4pi, double col, d3 r1, d3 r2, d3 r, d3 g, d3& Rb, d3& Rpb) {
  Rb = Rpb = mk3(0, 0, 0);
  const d3 R = r1 - r, Rp = r2 - r;
  const double a = sqrt(dot3(R, R)), b = sqrt(dot3(Rp, Rp));
  const double RRp = dot3(R, Rp);
  if (a < 1e-8 || b < 1e-8) return;
  const double P = a * b;
  if (fabs(RRp / P - 1.0) < 2.0 * col) {
    const double cref = __ddiv_rn(__ddiv_rn(RRp, a), b);
    if (fabs(cref - 1.0) < col) return;
  }
  const double Q = P + RRp;
  const double s = f4pi * (a + b) / (P * Q);
  const d3 C = cross3(R, Rp);
  const d3 Cb = g * s;
  const double sb = dot3(g, C);
  // s = f4pi S / (P Q): dS = s/S, dP = -s/P, dQ = -s/Q
  const double Sb = sb * s / (a + b);
  double Pb = -sb * s / P;
  const double Qb = -sb * s / Q;
  Pb += Qb;                 // Q = P + R.R'
  const double RRpb = Qb;
  const double abar = Sb + Pb * b, bbar = Sb + Pb * a;
  Rb = cross3(Rp, Cb) + R * (abar / a) + Rp * RRpb;
  Rpb = cross3(Cb, R) + Rp * (bbar / b) + R * RRpb;
}

constexpr int kVT = 128;   // threads per block and tile length

// Pass A: per target k, x_bar_k -= sum_m (Rb + Rpb) over the segments
// (r = x_k enters R and R' with a minus sign); skip rule of
// calculate_vs_shift (src/tangle.c:567-569).
__global__ void __launch_bounds__(kVT) k_bs_vjp_targets(double f4pi, double col, const double* __restrict__ pos,
                                                        const int2* __restrict__ links,
                                                        const int2* __restrict__ status,
                                                        const double* __restrict__ gnl, double* xbar,
                                                        int n, int chunk) {
  __shared__ double sh[kVT][6];
  __shared__ int sid[kVT][2];
  const int s_lo = blockIdx.y * chunk, s_hi = min(n, s_lo + chunk);   // this block's sources
  const int k = blockIdx.x * kVT + threadIdx.x;
  const bool act = k < n && status[k].x == OV_FREE;
  const d3 r = act ? ld3(pos, k) : mk3(0, 0, 0);
  const d3 g = act ? ld3(gnl, k) : mk3(0, 0, 0);
  d3 acc = mk3(0, 0, 0);
  for (int base = s_lo; base < s_hi; base += kVT) {
    __syncthreads();
    const int m = base + threadIdx.x;
    int f = -1;
    if (m < s_hi && status[m].x != OV_EMPTY) f = links[m].x;
    d3 a = mk3(0, 0, 0), b = a;
    if (f >= 0) {
      a = ld3(pos, m);
      b = ld3(pos, f);
    }
    sh[threadIdx.x][0] = a.x; sh[threadIdx.x][1] = a.y; sh[threadIdx.x][2] = a.z;
    sh[threadIdx.x][3] = b.x; sh[threadIdx.x][4] = b.y; sh[threadIdx.x][5] = b.z;
    sid[threadIdx.x][0] = m;
    sid[threadIdx.x][1] = f;
    __syncthreads();
    if (!act) continue;
    const int cnt = min(kVT, s_hi - base);
    for (int q = 0; q < cnt; ++q) {
      const int id = sid[q][0], fw = sid[q][1];
      if (fw < 0 || id == k || fw == k) continue;
      d3 Rb, Rpb;
      seg_vjp(f4pi, col, mk3(sh[q][0], sh[q][1], sh[q][2]), mk3(sh[q][3], sh[q][4], sh[q][5]), r, g, Rb, Rpb);
      acc = acc - (Rb + Rpb);
    }
  }
  if (act) {
    atomicAdd(&xbar[3 * (size_t)k], acc.x);
    atomicAdd(&xbar[3 * (size_t)k + 1], acc.y);
    atomicAdd(&xbar[3 * (size_t)k + 2], acc.z);
  }
}

// Pass B: per segment m (x_m -> x_fwd), sum over the targets of Rb (to x_m)
// and Rpb (to x_fwd).
__global__ void __launch_bounds__(kVT) k_bs_vjp_segments(double f4pi, double col, const double* __restrict__ pos,
                                                         const int2* __restrict__ links,
                                                         const int2* __restrict__ status,
                                                         const double* __restrict__ gnl, double* xbar,
                                                         int n, int chunk) {
  __shared__ double sh[kVT][6];   // target position and its cotangent
  __shared__ int sid[kVT];
  const int t_lo = blockIdx.y * chunk, t_hi = min(n, t_lo + chunk);   // this block's targets
  const int m = blockIdx.x * kVT + threadIdx.x;
  int f = -1;
  if (m < n && status[m].x != OV_EMPTY) f = links[m].x;
  const d3 r1 = f >= 0 ? ld3(pos, m) : mk3(0, 0, 0);
  const d3 r2 = f >= 0 ? ld3(pos, f) : mk3(0, 0, 0);
  d3 a1 = mk3(0, 0, 0), a2 = a1;
  for (int base = t_lo; base < t_hi; base += kVT) {
    __syncthreads();
    const int k = base + threadIdx.x;
    const bool t_ok = k < t_hi && status[k].x == OV_FREE;
    const d3 r = t_ok ? ld3(pos, k) : mk3(0, 0, 0);
    const d3 g = t_ok ? ld3(gnl, k) : mk3(0, 0, 0);
    sh[threadIdx.x][0] = r.x; sh[threadIdx.x][1] = r.y; sh[threadIdx.x][2] = r.z;
    sh[threadIdx.x][3] = g.x; sh[threadIdx.x][4] = g.y; sh[threadIdx.x][5] = g.z;
    sid[threadIdx.x] = t_ok ? k : -1;
    __syncthreads();
    if (f < 0) continue;
    const int cnt = min(kVT, t_hi - base);
    for (int q = 0; q < cnt; ++q) {
      const int kk = sid[q];
      if (kk < 0 || kk == m || kk == f) continue;
      d3 Rb, Rpb;
      seg_vjp(f4pi, col, r1, r2, mk3(sh[q][0], sh[q][1], sh[q][2]), mk3(sh[q][3], sh[q][4], sh[q][5]), Rb, Rpb);
      a1 = a1 + Rb;
      a2 = a2 + Rpb;
    }
  }
  if (f >= 0) {
    atomicAdd(&xbar[3 * (size_t)m], a1.x);
    atomicAdd(&xbar[3 * (size_t)m + 1], a1.y);
    atomicAdd(&xbar[3 * (size_t)m + 2], a1.z);
    atomicAdd(&xbar[3 * (size_t)f], a2.x);
    atomicAdd(&xbar[3 * (size_t)f + 1], a2.y);
    atomicAdd(&xbar[3 * (size_t)f + 2], a2.z);
  }
}

// out = a * x (+ out if accumulate), 3n doubles
__global__ void k_scale(const double* x, double a, double* out, int m, int accumulate) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  out[i] = accumulate ? out[i] + a * x[i] : a * x[i];
}

}  // namespace

bool ov_capture_params(const tangle_state* t, OvParams& P);

struct ov_adjoint {
  ov_state_impl s;
  tangle_state hdr;
  int n = 0;
  double vn[3] = {0, 0, 0};
  // trajectory of the last forward run: its normal-fluid vector and
  // precision are kept apart from vn, which velocity calls overwrite
  double t0 = 0, dt = 0, fwd_vn[3] = {0, 0, 0};
  int nsteps = 0, every = 1, classic = 0, have_fwd = 0, fwd_precision = 0;
  unsigned long long generation = 0;
  DevBuf ckpt, blk, y[3], kv[3], kbar[4], xbar, ybar, gnl, vnbar, vn_dev, gv, tmp_dxi, tmp_tan,
      tmp_nrm, tmp_vs, tmp_v;
};

namespace {

int blocks(long long m, int t = 256) { return (int)((m + t - 1) / t); }

// all-pairs passes: split the inner range so that a small tangle still
// fills the GPU (about 4 blocks per SM); returns the range per split
int pair_chunk(int n, int* splits) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 1;
  }
  const int bx = blocks(n, kVT);
  int sp = std::min(32, std::max(1, (4 * sms + bx - 1) / bx));
  int chunk = (n + sp - 1) / sp;
  chunk = (chunk + kVT - 1) / kVT * kVT;
  *splits = std::max(1, (n + chunk - 1) / chunk);
  return chunk;
}

bool flow_ok(const OvFlow& f) { return f.kind == OVF_NONE || f.kind == OVF_SIMPLE; }

// parameters of the current globals, with the normal-fluid vector of the
// run and the direct sum
bool refresh(ov_adjoint* a) {
  OvParams& P = a->s.P;
  if (!ov_capture_params(&a->hdr, P)) return false;
  P.n_img = 0;
  P.use_bh = 0;
  if (!flow_ok(P.vs) || (P.use_mf && !flow_ok(P.vn))) {
    ov_set_error(OV_ERR_FLOW, "adjoint: superfluid and normal-fluid flows must be 'no flow' or 'simple'");
    return false;
  }
  P.vn.kind = OVF_SIMPLE;
  for (int c = 0; c < 3; ++c) P.vn.v[0][c] = a->vn[c];
  return true;
}

LocalP local_params(const OvParams& P) {
  LocalP L;
  L.kappa = P.kappa;
  L.core_a = P.core_a;
  L.alpha = P.alpha;
  L.alpha_p = P.alpha_p;
  L.hyperalpha = P.hyperalpha;
  L.curv_thr = P.max_curv / P.dl_max;
  for (int c = 0; c < 3; ++c) L.vs_flow[c] = P.vs.kind == OVF_SIMPLE ? P.vs.v[0][c] : 0.0;
  L.use_mf = P.use_mf;
  L.hyperfriction = P.hyperfriction;
  L.lia_only = P.lia_only;
  return L;
}

// velocities at positions x (3n doubles, device) into v
bool velocity_at(ov_adjoint* a, const double* x, double t, double* v) {
  ov_state_impl* s = &a->s;
  return ov_geometry(s, x, a->tmp_dxi.as<double>(), a->tmp_tan.as<double>(), a->tmp_nrm.as<double>()) &&
         ov_velocities(s, t, x, a->tmp_dxi.as<double>(), a->tmp_tan.as<double>(), a->tmp_nrm.as<double>(), v,
                       a->tmp_vs.as<double>(), nullptr);
}

// y_bar (zeroed here) = (dv/dx at x)^T g; vn_bar accumulates
bool velocity_vjp(ov_adjoint* a, const double* x, const double* g, double* ybar) {
  ov_state_impl* s = &a->s;
  const int n = a->n;
  const size_t v3 = sizeof(double) * 3 * (size_t)n;
  OV_TRY_CUDA(cudaMemsetAsync(ybar, 0, v3, s->stream));
  OV_TRY_CUDA(cudaMemsetAsync(a->gnl.p, 0, v3, s->stream));
  double* vnl = s->v_nl.as<double>();
  if (s->P.lia_only) {
    OV_TRY_CUDA(cudaMemsetAsync(vnl, 0, v3, s->stream));
  } else if (!ov_direct_nodes(s, x, vnl, s->v_img.as<double>())) {
    return false;
  }
  const LocalP L = local_params(s->P);
  k_local_vjp<<<blocks((long long)n * kLocalInputs), 256, 0, s->stream>>>(
      L, x, s->links.as<int2>(), s->status.as<int2>(), vnl, a->vn_dev.as<double>(), g, ybar,
      a->gnl.as<double>(), a->vnbar.as<double>(), n);
  OV_LAUNCHED();
  if (!s->P.lia_only) {
    int splits = 1;
    const int chunk = pair_chunk(n, &splits);
    const dim3 grid(blocks(n, kVT), splits);
    k_bs_vjp_targets<<<grid, kVT, 0, s->stream>>>(s->P.f4pi, s->P.col_cut, x, s->links.as<int2>(), s->status.as<int2>(),
                                                  a->gnl.as<double>(), ybar, n, chunk);
    OV_LAUNCHED();
    k_bs_vjp_segments<<<grid, kVT, 0, s->stream>>>(s->P.f4pi, s->P.col_cut, x, s->links.as<int2>(), s->status.as<int2>(),
                                                   a->gnl.as<double>(), ybar, n, chunk);
    OV_LAUNCHED();
  }
  OV_TRY_CUDA(cudaGetLastError());
  return true;
}

bool scale(ov_adjoint* a, const double* x, double c, double* out, bool acc) {
  const int m = 3 * a->n;
  k_scale<<<blocks(m), 256, 0, a->s.stream>>>(x, c, out, m, acc ? 1 : 0);
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  return true;
}

// one RK4 step (update_tangle + rk4_step) on the state's positions at time t
bool forward_step(ov_adjoint* a, double t) {
  ov_state_impl* s = &a->s;
  return velocity_at(a, s->pos.as<double>(), t, s->vels.as<double>()) && ov_rk4(s, t, a->dt, a->classic);
}

// Reverse of one step from x0 at time t: x_bar (the step's output cotangent
// on entry) becomes the input cotangent.
bool reverse_step(ov_adjoint* a, const double* x0, double t) {
  ov_state_impl* s = &a->s;
  const double dt = a->dt;
  const double h[3] = {dt / 2, dt / 2, a->classic ? dt : dt / 2};
  const double ts[4] = {t, t + dt / 2, t + dt / 2, t + dt};
  const int2* st = s->status.as<int2>();
  double* xb = a->xbar.as<double>();
  // stage positions y1..y3 (k1..k3 recomputed)
  const double* ys[4] = {x0, a->y[0].as<double>(), a->y[1].as<double>(), a->y[2].as<double>()};
  for (int q = 0; q < 3; ++q) {
    if (!velocity_at(a, ys[q], ts[q], a->kv[q].as<double>())) return false;
    if (!ov_launch_euler(s->stream, st, x0, a->kv[q].as<double>(), h[q], a->y[q].as<double>(), a->n))
      return false;
  }
  // x1 = x0 + dt/6 k1 + dt/3 k2 + dt/3 k3 + dt/6 k4
  const double w[4] = {dt / 6, dt / 3, dt / 3, dt / 6};
  for (int q = 0; q < 4; ++q)
    if (!scale(a, xb, w[q], a->kbar[q].as<double>(), false)) return false;
  // stage q (k_{q+1} = v(y_q), y_q = x0 + h_{q-1} k_q): back to front
  for (int q = 3; q >= 0; --q) {
    if (!velocity_vjp(a, ys[q], a->kbar[q].as<double>(), a->ybar.as<double>())) return false;
    if (!scale(a, a->ybar.as<double>(), 1.0, xb, true)) return false;
    if (q > 0 && !scale(a, a->ybar.as<double>(), h[q - 1], a->kbar[q - 1].as<double>(), true)) return false;
  }
  return true;
}

bool reserve_all(ov_adjoint* a) {
  const size_t v3 = sizeof(double) * 3 * (size_t)std::max(1, a->n);
  DevBuf* bufs[] = {&a->y[0], &a->y[1], &a->y[2], &a->kv[0], &a->kv[1], &a->kv[2], &a->kbar[0], &a->kbar[1],
                    &a->kbar[2], &a->kbar[3], &a->xbar, &a->ybar, &a->gnl, &a->gv, &a->tmp_tan,
                    &a->tmp_nrm, &a->tmp_vs, &a->tmp_v};
  for (DevBuf* b : bufs)
    if (!b->reserve(v3)) return false;
  return a->tmp_dxi.reserve(sizeof(double) * std::max(1, a->n)) && a->vnbar.reserve(64) &&
         a->vn_dev.reserve(64);
}

bool set_vn(ov_adjoint* a, const double* vn) {
  if (vn)
    for (int c = 0; c < 3; ++c) a->vn[c] = vn[c];
  if (!refresh(a)) return false;
  OV_TRY_CUDA(cudaMemcpyAsync(a->vn_dev.p, a->vn, sizeof(double) * 3, cudaMemcpyHostToDevice, a->s.stream));
  return true;
}

bool upload_pos(ov_adjoint* a, const double* x, double* dst) {
  if (!x) {
    ov_set_error(OV_ERR_INVALID, "adjoint: positions missing");
    return false;
  }
  OV_TRY_CUDA(cudaMemcpyAsync(dst, x, sizeof(double) * 3 * a->n, cudaMemcpyHostToDevice, a->s.stream));
  return true;
}

bool sync_to(ov_adjoint* a, double* host, const double* dev, size_t count) {
  if (host) OV_TRY_CUDA(cudaMemcpyAsync(host, dev, sizeof(double) * count, cudaMemcpyDeviceToHost, a->s.stream));
  OV_TRY_CUDA(cudaStreamSynchronize(a->s.stream));
  return true;
}

}  // namespace

extern "C" {

ov_adjoint* ov_adjoint_create(const struct tangle_state* t) {
  ov_clear_error();
  if (!t || t->N <= 0 || !t->status || !t->connections || !t->vnodes) {
    ov_set_error(OV_ERR_INVALID, "ov_adjoint_create: empty tangle");
    return nullptr;
  }
  for (int w = 0; w < 6; ++w)
    if (t->box.wall[w] != WALL_OPEN) {
      ov_set_error(OV_ERR_INVALID, "ov_adjoint_create: open boundaries only (wall %d)", w);
      return nullptr;
    }
  if (t->bimg.n != 0) {
    ov_set_error(OV_ERR_INVALID, "ov_adjoint_create: no boundary images");
    return nullptr;
  }
  for (int k = 0; k < t->N; ++k) {
    const int st = t->status[k].status;
    if (st == EMPTY) continue;
    const int f = t->connections[k].forward, r = t->connections[k].reverse;
    if (st != FREE || f < 0 || r < 0 || f >= t->N || r >= t->N || t->status[f].status != FREE ||
        t->status[r].status != FREE || t->connections[f].reverse != k || t->connections[r].forward != k) {
      ov_set_error(OV_ERR_INVALID, "ov_adjoint_create: node %d is not a free node of a closed loop", k);
      return nullptr;
    }
  }
  ov_adjoint* a = new ov_adjoint();
  a->hdr = *t;
  a->hdr.N = 0;
  a->hdr.vnodes = nullptr;
  a->n = t->N;
  bool ok = ov_upload_tangle(&a->s, t) && reserve_all(a);
  if (ok) {
    // the normal-fluid vector of vn_conf when it is "simple"
    if (a->s.P.vn.kind == OVF_SIMPLE)
      for (int c = 0; c < 3; ++c) a->vn[c] = a->s.P.vn.v[0][c];
    ok = set_vn(a, nullptr) && sync_to(a, nullptr, nullptr, 0);
  }
  if (!ok) {
    const int e = ov_last_error();
    ov_adjoint_destroy(a);
    if (!ov_last_error()) ov_set_error(e ? e : OV_ERR_CUDA, "ov_adjoint_create failed");
    return nullptr;
  }
  return a;
}

void ov_adjoint_destroy(ov_adjoint* a) {
  if (!a) return;
  DevBuf* bufs[] = {&a->ckpt, &a->blk, &a->y[0], &a->y[1], &a->y[2], &a->kv[0], &a->kv[1], &a->kv[2],
                    &a->kbar[0], &a->kbar[1], &a->kbar[2], &a->kbar[3], &a->xbar, &a->ybar, &a->gnl,
                    &a->vnbar, &a->vn_dev, &a->gv, &a->tmp_dxi, &a->tmp_tan, &a->tmp_nrm, &a->tmp_vs,
                    &a->tmp_v};
  for (DevBuf* b : bufs) b->release();
  ov_state_impl* s = &a->s;
  DevBuf* sb[] = {&s->pos, &s->links, &s->status, &s->dxi, &s->tan, &s->nrm, &s->vels, &s->vs, &s->pos0,
                  &s->spos, &s->sdxi, &s->stan, &s->snrm, &s->svs, &s->k2, &s->k3, &s->k4, &s->v_nl,
                  &s->v_img, &s->img_part, &s->seg64, &s->segid, &s->dflag};
  for (DevBuf* b : sb) b->release();
  ov_tree_release(&s->tree);
  if (s->stream) cudaStreamDestroy(s->stream);
  if (s->ev0) cudaEventDestroy(s->ev0);
  if (s->ev1) cudaEventDestroy(s->ev1);
  if (s->ev2) cudaEventDestroy(s->ev2);
  delete a;
}

int ov_adjoint_velocity(ov_adjoint* a, const double* x, const double* vn, double t, double* v) {
  ov_clear_error();
  if (!a || !v) { ov_set_error(OV_ERR_INVALID, "null adjoint or output"); return ov_last_error(); }
  if (!set_vn(a, vn) || !upload_pos(a, x, a->ybar.as<double>()) ||
      !velocity_at(a, a->ybar.as<double>(), t, a->tmp_v.as<double>()) ||
      !sync_to(a, v, a->tmp_v.as<double>(), 3 * (size_t)a->n))
    return ov_last_error();
  return OV_OK;
}

int ov_adjoint_velocity_vjp(ov_adjoint* a, const double* x, const double* vn, double t, const double* v_bar,
                            double* x_bar, double* vn_bar) {
  ov_clear_error();
  (void)t;
  if (!a || !v_bar || !x_bar) { ov_set_error(OV_ERR_INVALID, "null adjoint or array"); return ov_last_error(); }
  ov_state_impl* s = &a->s;
  bool ok = set_vn(a, vn) && upload_pos(a, x, a->y[0].as<double>()) &&
            upload_pos(a, v_bar, a->gv.as<double>()) &&
            ov_cuda_ok(cudaMemsetAsync(a->vnbar.p, 0, 64, s->stream), "cudaMemsetAsync") &&
            velocity_vjp(a, a->y[0].as<double>(), a->gv.as<double>(), a->ybar.as<double>()) &&
            sync_to(a, x_bar, a->ybar.as<double>(), 3 * (size_t)a->n) &&
            sync_to(a, vn_bar, a->vnbar.as<double>(), vn_bar ? 3 : 0);
  return ok ? OV_OK : ov_last_error();
}

int ov_adjoint_forward(ov_adjoint* a, const double* x0, const double* vn, double t0, double dt, int nsteps,
                       int every, double* x_final) {
  ov_clear_error();
  if (!a || nsteps < 0 || every < 1) {
    ov_set_error(OV_ERR_INVALID, "ov_adjoint_forward: null adjoint, negative steps or checkpoint interval < 1");
    return ov_last_error();
  }
  ov_state_impl* s = &a->s;
  a->have_fwd = 0;
  a->t0 = t0;
  a->dt = dt;
  a->nsteps = nsteps;
  a->every = every;
  a->classic = ov_get_rk4_classic();
  const size_t v3 = 3 * (size_t)a->n;
  const int n_ckpt = (nsteps + every - 1) / every;
  if (!set_vn(a, vn) || !upload_pos(a, x0, s->pos.as<double>()) ||
      !a->ckpt.reserve(sizeof(double) * v3 * std::max(1, n_ckpt)) ||
      !a->blk.reserve(sizeof(double) * v3 * every))
    return ov_last_error();
  for (int i = 0; i < nsteps; ++i) {
    if (i % every == 0 &&
        !ov_cuda_ok(cudaMemcpyAsync(a->ckpt.as<double>() + v3 * (i / every), s->pos.p, sizeof(double) * v3,
                                    cudaMemcpyDeviceToDevice, s->stream),
                    "cudaMemcpyAsync"))
      return ov_last_error();
    if (!forward_step(a, t0 + i * dt)) return ov_last_error();
  }
  if (!sync_to(a, x_final, s->pos.as<double>(), v3)) return ov_last_error();
  for (int c = 0; c < 3; ++c) a->fwd_vn[c] = a->vn[c];
  a->fwd_precision = s->P.precision;
  a->have_fwd = 1;
  ++a->generation;
  return OV_OK;
}

int ov_adjoint_backward(ov_adjoint* a, const double* x_final_bar, double* x0_bar, double* vn_bar) {
  ov_clear_error();
  if (!a || !a->have_fwd || !x_final_bar) {
    ov_set_error(OV_ERR_INVALID, "ov_adjoint_backward: no forward run or no cotangent");
    return ov_last_error();
  }
  ov_state_impl* s = &a->s;
  const size_t v3 = 3 * (size_t)a->n;
  // recompute with the forward run's vn and precision, whatever velocity
  // calls or precision changes came in between
  if (!set_vn(a, a->fwd_vn)) return ov_last_error();
  s->P.precision = a->fwd_precision;
  if (!upload_pos(a, x_final_bar, a->xbar.as<double>()) ||
      !ov_cuda_ok(cudaMemsetAsync(a->vnbar.p, 0, 64, s->stream), "cudaMemsetAsync"))
    return ov_last_error();
  const int n_ckpt = (a->nsteps + a->every - 1) / a->every;
  for (int c = n_ckpt - 1; c >= 0; --c) {
    const int i0 = c * a->every, i1 = std::min(a->nsteps, i0 + a->every);
    // recompute the block's step start positions from its checkpoint
    if (!ov_cuda_ok(cudaMemcpyAsync(s->pos.p, a->ckpt.as<double>() + v3 * c, sizeof(double) * v3,
                                    cudaMemcpyDeviceToDevice, s->stream),
                    "cudaMemcpyAsync"))
      return ov_last_error();
    for (int i = i0; i < i1; ++i) {
      if (!ov_cuda_ok(cudaMemcpyAsync(a->blk.as<double>() + v3 * (i - i0), s->pos.p, sizeof(double) * v3,
                                      cudaMemcpyDeviceToDevice, s->stream),
                      "cudaMemcpyAsync"))
        return ov_last_error();
      if (i + 1 < i1 && !forward_step(a, a->t0 + i * a->dt)) return ov_last_error();
    }
    for (int i = i1 - 1; i >= i0; --i)
      if (!reverse_step(a, a->blk.as<double>() + v3 * (i - i0), a->t0 + i * a->dt)) return ov_last_error();
  }
  if (!sync_to(a, x0_bar, a->xbar.as<double>(), v3) || !sync_to(a, vn_bar, a->vnbar.as<double>(), vn_bar ? 3 : 0))
    return ov_last_error();
  return OV_OK;
}

unsigned long long ov_adjoint_generation(const ov_adjoint* a) { return a ? a->generation : 0; }

}  // extern "C"
