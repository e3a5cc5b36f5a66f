// ov_geom.cu - per-node kernels: arc lengths, 4-point tangent/normal
// stencils, the velocity epilogue (local induction, external flow,
// hyperfriction, mutual friction, slip) and the RK4 stage arithmetic.
// All FP64; each thread owns one node slot.  HBM-bound: ~150 B per node.
#include "ov_internal.h"
#include "ov_links.cuh"
#include "ov_node.cuh"

namespace {

constexpr int kThreads = 256;

// idx: the slots to compute (null: slots 0 .. n-1)
__global__ void k_dxi(OvParams P, Links L, const double* __restrict__ pos, double* dxi,
                      const int* __restrict__ idx, int n, int* flag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k = idx ? idx[i] : i;
  if (L.st[k].x == OV_EMPTY) return;
  double d;
  if (!dxi_node(P, L, pos, k, d)) { atomicOr(flag, 1); return; }
  dxi[k] = d;
}

// pass 0: pinned and ordinary nodes; pass 1: nodes next to a pinned node,
// which use their neighbours' tangents (src/tangle.c:366-430)
__global__ void k_tangents(OvParams P, Links L, const double* __restrict__ pos,
                           const double* __restrict__ dxi, double* tan, double* nrm,
                           const int* __restrict__ idx, int n, int pass, int* flag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k = idx ? idx[i] : i;
  int2 st = L.st[k];
  if (st.x == OV_EMPTY) return;
  if ((pass == 1) != near_pinned(L, k)) return;
  d3 t, nn;
  auto arc = [&](int kk, int dist, double& out) { return arc_length(L, dxi, kk, dist, out); };
  if (!tangent_node(P, L, pos, k, arc, tan, t, nn)) { atomicOr(flag, 1); return; }
  st3(tan, k, t);
  st3(nrm, k, nn);
}

// velocity assembly per node (update_velocity, src/tangle.c:583-684)
// time = t0 + (*t_dev when given: a graph replayed at advancing times)
__global__ void k_epilogue(OvParams P, Links L, const double* __restrict__ t_dev, double t0,
                           const double* __restrict__ pos, const double* __restrict__ tan,
                           const double* __restrict__ nrm, const double* __restrict__ v_nl,
                           const double* __restrict__ v_img, double* vels, double* vs_out, int k0,
                           int k1, const int* __restrict__ idx, int* flag) {
  const int i = k0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= k1) return;
  const int k = idx ? idx[i] : i;
  const double t = t_dev ? t0 + *t_dev : t0;
  if (L.st[k].x == OV_EMPTY) return;
  const d3 vnl = P.lia_only ? mk3(0, 0, 0) : ld3(v_nl, k);
  const d3 vim = (P.lia_only || P.n_img == 0) ? mk3(0, 0, 0) : ld3(v_img, k);
  d3 v, vs;
  const int err = epilogue_node(P, L, t, pos, k, ld3(tan, k), ld3(nrm, k), vnl, vim, v, vs);
  if (err & 1) { atomicOr(flag, 1); return; }
  if (err) atomicOr(flag, err);
  st3(vs_out, k, vs);
  st3(vels, k, v);
}

// x_s = x_0 + h v  (euler_step2, src/vortex_dynamics.c:36-52)
__global__ void k_euler(const int2* __restrict__ st, const double* __restrict__ x0,
                        const double* __restrict__ v, double h, double* xs, int n) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n || st[k].x == OV_EMPTY) return;
#pragma unroll
  for (int c = 0; c < 3; ++c) xs[3 * k + c] = x0[3 * k + c] + v[3 * k + c] * h;
}

// x += dt/6 k1 + dt/3 k2 + dt/3 k3 + dt/6 k4 (src/vortex_dynamics.c:94-112)
__global__ void k_rk4_combine(const int2* __restrict__ st, const double* __restrict__ k1,
                              const double* __restrict__ k2, const double* __restrict__ k3,
                              const double* __restrict__ k4, double dt, double* x, int n) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n || st[k].x == OV_EMPTY) return;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    int i = 3 * k + c;
    double mv = k1[i] * (dt / 6);
    mv += k2[i] * (dt / 3);
    mv += k3[i] * (dt / 3);
    mv += k4[i] * (dt / 6);
    x[i] += mv;
  }
}

int blocks_for(int n) { return (n + kThreads - 1) / kThreads; }

}  // namespace

// ---------------------------------------------------------------- launchers
// Kernel launches only (no host synchronisation, so they can be captured in
// a CUDA graph); link and finiteness errors accumulate in *flag.

bool ov_launch_geometry(cudaStream_t st, const OvParams& P, const int2* links, const int2* status,
                        const double* pos, double* dxi, double* tan, double* nrm, int n, int* flag) {
  if (n <= 0) return true;
  return ov_launch_geometry_list(st, P, links, status, pos, dxi, tan, nrm, nullptr, n, flag);
}

bool ov_launch_geometry_list(cudaStream_t st, const OvParams& P, const int2* links, const int2* status,
                             const double* pos, double* dxi, double* tan, double* nrm, const int* idx, int n,
                             int* flag) {
  if (n <= 0) return true;
  Links L{links, status};
  k_dxi<<<blocks_for(n), kThreads, 0, st>>>(P, L, pos, dxi, idx, n, flag);
  OV_LAUNCHED();
  k_tangents<<<blocks_for(n), kThreads, 0, st>>>(P, L, pos, dxi, tan, nrm, idx, n, 0, flag);
  OV_LAUNCHED();
  k_tangents<<<blocks_for(n), kThreads, 0, st>>>(P, L, pos, dxi, tan, nrm, idx, n, 1, flag);
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  return true;
}

bool ov_launch_epilogue(cudaStream_t st, const OvParams& P, const int2* links, const int2* status,
                        const double* t_dev, double t0, const double* pos, const double* tan,
                        const double* nrm, const double* v_nl, const double* v_img, double* vels,
                        double* vs, int k0, int k1, int* flag) {
  if (k1 <= k0) return true;
  Links L{links, status};
  k_epilogue<<<blocks_for(k1 - k0), kThreads, 0, st>>>(P, L, t_dev, t0, pos, tan, nrm, v_nl, v_img,
                                                         vels, vs, k0, k1, nullptr, flag);
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  return true;
}

bool ov_launch_epilogue_list(cudaStream_t st, const OvParams& P, const int2* links, const int2* status,
                             double t0, const double* pos, const double* tan, const double* nrm,
                             const double* v_nl, const double* v_img, double* vels, double* vs,
                             const int* idx, int count, int* flag) {
  if (count <= 0) return true;
  Links L{links, status};
  k_epilogue<<<blocks_for(count), kThreads, 0, st>>>(P, L, nullptr, t0, pos, tan, nrm, v_nl, v_img, vels,
                                                     vs, 0, count, idx, flag);
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  return true;
}

bool ov_launch_euler(cudaStream_t st, const int2* status, const double* x0, const double* v,
                     double h, double* xs, int n) {
  if (n <= 0) return true;
  k_euler<<<blocks_for(n), kThreads, 0, st>>>(status, x0, v, h, xs, n);
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  return true;
}

bool ov_launch_rk4_combine(cudaStream_t st, const int2* status, const double* k1, const double* k2,
                           const double* k3, const double* k4, double dt, double* x, int n) {
  if (n <= 0) return true;
  k_rk4_combine<<<blocks_for(n), kThreads, 0, st>>>(status, k1, k2, k3, k4, dt, x, n);
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  return true;
}

bool ov_flag_status(int h, const char* where) {
  if (h & 1) {
    ov_set_error(OV_ERR_INVALID, "%s: broken vortex links (a free node without a neighbour)", where);
    return false;
  }
  if (h & 2) {
    ov_set_error(OV_ERR_NONFINITE, "%s: non-finite velocity", where);
    return false;
  }
  return true;
}

static bool check_flag(ov_state_impl* s, const char* where) {
  int h = 0;
  OV_TRY_CUDA(cudaMemcpyAsync(&h, s->dflag.p, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  OV_TRY_CUDA(cudaStreamSynchronize(s->stream));
  return ov_flag_status(h, where);
}

bool ov_geometry(ov_state_impl* s, const double* pos, double* dxi, double* tan, double* nrm) {
  if (s->n == 0) return true;
  int* flag = s->dflag.as<int>();
  OV_TRY_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s->stream));
  if (!ov_launch_geometry(s->stream, s->P, s->links.as<int2>(), s->status.as<int2>(), pos, dxi, tan,
                          nrm, s->n, flag))
    return false;
  return check_flag(s, "update_tangents_normals");
}

bool ov_epilogue(ov_state_impl* s, double t, const double* pos, const double* tan,
                 const double* nrm, const double* v_nl, const double* v_img, double* vels,
                 double* vs, int k0, int k1) {
  if (k1 <= k0) return true;
  int* flag = s->dflag.as<int>();
  OV_TRY_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s->stream));
  if (!ov_launch_epilogue(s->stream, s->P, s->links.as<int2>(), s->status.as<int2>(), nullptr, t, pos,
                          tan, nrm, v_nl, v_img, vels, vs, k0, k1, flag))
    return false;
  return check_flag(s, "update_velocities");
}

bool ov_euler(ov_state_impl* s, double dt) {
  if (s->n == 0) return true;
  k_euler<<<blocks_for(s->n), kThreads, 0, s->stream>>>(s->status.as<int2>(), s->pos.as<double>(),
                                                         s->vels.as<double>(), dt,
                                                         s->pos.as<double>(), s->n);
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  return true;
}

// Stage q = 1..3 positions of rk4_step2 (src/vortex_dynamics.c:76-92):
// xs = x0 + h_q k_q, with k_1 = vels and k_2, k_3 the stage velocities; the
// steps h are dt/2, dt/2 and, for the last stage, dt/2 like the reference
// unless `classic` (dt).
bool ov_rk4_stage_positions(ov_state_impl* s, int q, double dt, int classic) {
  if (s->n == 0) return true;
  const double h[3] = {dt / 2, dt / 2, classic ? dt : dt / 2};
  double* x0 = s->pos.as<double>();
  double* xs = s->spos.as<double>();
  // EMPTY slots of the stage positions are never read, but keep them defined
  if (q == 1)
    OV_TRY_CUDA(cudaMemcpyAsync(xs, x0, sizeof(double) * 3 * s->n, cudaMemcpyDeviceToDevice, s->stream));
  const double* prev = q == 1 ? s->vels.as<double>() : (q == 2 ? s->k2.as<double>() : s->k3.as<double>());
  k_euler<<<blocks_for(s->n), kThreads, 0, s->stream>>>(s->status.as<int2>(), x0, prev, h[q - 1], xs,
                                                         s->n);
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  return true;
}

// x0 += dt/6 k1 + dt/3 k2 + dt/3 k3 + dt/6 k4 (src/vortex_dynamics.c:95-112)
bool ov_rk4_combine(ov_state_impl* s, double dt) {
  if (s->n == 0) return true;
  k_rk4_combine<<<blocks_for(s->n), kThreads, 0, s->stream>>>(
      s->status.as<int2>(), s->vels.as<double>(), s->k2.as<double>(), s->k3.as<double>(),
      s->k4.as<double>(), dt, s->pos.as<double>(), s->n);
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  return true;
}

// rk4_step2 (src/vortex_dynamics.c:58-117) on the device state.  Stage 4
// advances dt/2 like the reference unless `classic`.
bool ov_rk4(ov_state_impl* s, double t, double dt, int classic) {
  if (s->n == 0) return true;
  double* ks[3] = {s->k2.as<double>(), s->k3.as<double>(), s->k4.as<double>()};
  const double ts[3] = {t + dt / 2, t + dt / 2, t + dt};
  const double* xs = s->spos.as<double>();
  for (int q = 1; q <= 3; ++q) {
    if (!ov_rk4_stage_positions(s, q, dt, classic)) return false;
    if (!ov_geometry(s, xs, s->sdxi.as<double>(), s->stan.as<double>(), s->snrm.as<double>()))
      return false;
    if (!ov_velocities(s, ts[q - 1], xs, s->sdxi.as<double>(), s->stan.as<double>(),
                       s->snrm.as<double>(), ks[q - 1], s->svs.as<double>(), nullptr))
      return false;
  }
  return ov_rk4_combine(s, dt);
}
