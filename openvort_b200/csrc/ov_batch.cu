// ov_batch.cu - batched ensembles: many independent open-boundary systems
// (each a few closed loops) advanced together (ov_batch_*, include/
// openvort_b200.h).
//
// All systems share one slot array (system s in slots off[s] .. off[s+1]-1,
// links inside the system), so the per-node kernels of a single tangle
// (arc lengths, tangents/normals, epilogue, RK4 stage arithmetic) run over
// the whole ensemble unchanged.  Only the Biot-Savart sum is block-diagonal:
// a target sums the segments of its own system (the loop of update_velocity,
// src/tangle.c:611-619, over that system's tangle).
//
// The sum is one persistent kernel per RK4 stage.  Work items are (system,
// block of consecutive targets), the largest systems first; each resident
// block takes the next item from a counter, stages its system's segments
// through shared memory and sweeps them for its targets.  One RK4 step
// (update_tangle + rk4_step: 4 evaluations) is captured once as a CUDA graph
// and replayed; the time of each stage is read from device memory so the
// same graph serves every step.
#include <algorithm>
#include <vector>

#include "ov_internal.h"
#include "ov_pair.cuh"

namespace {

struct BatchView {
  const int* off;       // n_sys + 1 slot offsets
  const int2* items;    // (system, first target slot), costliest first
  const double* near2;  // per system: FP64 within this squared distance (mixed form)
  int n_items;
};

// far dummy for slots without a segment: a zero-length segment at (1e4)^3,
// which every formula here evaluates to exactly zero
constexpr double kNoSeg = 1.0e4;

// What a Biot-Savart kernel does with a target's sum (inactive targets:
// EMPTY slots, whose sums are zero): v_nl for the per-node kernels that
// follow.
struct StoreSums {
  double* v_nl;
  __device__ void operator()(const OvParams&, int k, bool act, d3 v) const {
    st3(v_nl, k, act ? v : mk3(0, 0, 0));
  }
};

// FP64 form: the reference's formula and cut-offs for every pair.  The
// skip rule of calculate_vs_shift (src/tangle.c:567-569) is implied here:
// with open boundaries the two segments it skips have an endpoint at the
// target itself, where the |R| < 1e-8 cut-off returns zero.
template <int TB, int TS>
__global__ void __launch_bounds__(TB) k_batch_bs64(OvParams P, BatchView B,
                                                   const double* __restrict__ pos,
                                                   const int2* __restrict__ links,
                                                   const int2* __restrict__ status,
                                                   StoreSums out, int* __restrict__ work) {
  __shared__ double sh_r[TS][6];
  __shared__ int sh_item;
  for (;;) {
    __syncthreads();   // the previous item's tile reads and sh_item reads are done
    if (threadIdx.x == 0) sh_item = atomicAdd(work, 1);
    __syncthreads();
    const int it = sh_item;
    if (it >= B.n_items) return;   // uniform over the block
    const int2 w = B.items[it];
    const int s0 = B.off[w.x], s1 = B.off[w.x + 1];
    const int k = w.y + threadIdx.x;
    const bool act = k < s1 && status[k].x == OV_FREE;
    const d3 r = act ? ld3(pos, k) : mk3(0, 0, 0);
    double ax = 0, ay = 0, az = 0;
    for (int base = s0; base < s1; base += TS) {
      __syncthreads();
      for (int q = threadIdx.x; q < TS; q += TB) {
        const int m = base + q;
        d3 a = mk3(kNoSeg, kNoSeg, kNoSeg), b = a;
        if (m < s1 && status[m].x != OV_EMPTY) {
          const int f = links[m].x;
          if (f >= 0) {
            a = ld3(pos, m);
            b = ld3(pos, f);
          }
        }
        sh_r[q][0] = a.x; sh_r[q][1] = a.y; sh_r[q][2] = a.z;
        sh_r[q][3] = b.x; sh_r[q][4] = b.y; sh_r[q][5] = b.z;
      }
      __syncthreads();
      if (act) {
        const int cnt = min(TS, s1 - base);
        for (int q = 0; q < cnt; ++q) {
          const d3 v = seg_vel64(P.f4pi, mk3(sh_r[q][0], sh_r[q][1], sh_r[q][2]),
                                 mk3(sh_r[q][3], sh_r[q][4], sh_r[q][5]), r);
          ax += v.x; ay += v.y; az += v.z;
        }
      }
    }
    if (k < s1) out(P, k, act, mk3(ax, ay, az));
  }
}

// Mixed form: FP32 offsets from one origin per work item.  Items of 64
// threads (128 targets at two per thread) take single-rounded offsets from
// the item's middle target: the items span at most 64 node spacings either
// side, and the
// measured error against the FP64 form is 3.8e-6 on the 4096-system bench
// ensemble.  Larger items take two-float offsets (hi + lo) from their first
// target (error 8e-8), since a single rounding over a whole ring would cost a
// near segment ~1e-6 of its |R|.  Two sources per
// f32x2 instruction and kTT targets per thread (pair_interact); pairs
// nearer than max(4 |ds|, the system's near radius) or too close to the
// colinearity cut-off take the FP64 formula from the FP64 positions.  FP32
// partial sums over 32 sources are added into FP64 sums.  With open
// boundaries the two segments the skip rule drops have an endpoint at the
// target, so they are near and the FP64 cut-off returns zero for them.
template <int TB, int TS, bool kTwo = (TB > 64)>
__global__ void __launch_bounds__(TB) k_batch_bs_mixed(OvParams P, BatchView B,
                                                       const double* __restrict__ pos,
                                                       const int2* __restrict__ links,
                                                       const int2* __restrict__ status,
                                                       StoreSums out, int* __restrict__ work) {
  static_assert(TS % 32 == 0, "sources per tile");
  __shared__ PairSrc<kTwo> sh[TS / 2];
  __shared__ int sh_item;
  const double f4pi = P.f4pi;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) sh_item = atomicAdd(work, 1);
    __syncthreads();
    const int it = sh_item;
    if (it >= B.n_items) return;
    const int2 w = B.items[it];
    const int s0 = B.off[w.x], s1 = B.off[w.x + 1];
    const double near2 = B.near2[w.x];
    // two-float offsets from the item's first target; single-rounded ones
    // from its middle target
    const d3 O = ld3(pos, kTwo ? w.y : w.y + min(TB * kTT, s1 - w.y) / 2);
    int kk[kTT];
    PairTargets T;
    double acc[kTT][3];
#pragma unroll
    for (int u = 0; u < kTT; ++u) {
      const int k = w.y + threadIdx.x + TB * u;
      const bool act = k < s1 && status[k].x == OV_FREE;
      kk[u] = act ? k : -1;
      const d3 r = act ? ld3(pos, k) : O;
      set_target(T, u, r.x - O.x, r.y - O.y, r.z - O.z);
      acc[u][0] = acc[u][1] = acc[u][2] = 0;
    }
    auto special = [&](int u, int id) {
#pragma unroll
      for (int v = 0; v < kTT; ++v) {
        if (v != u) continue;
        const int k = kk[v];
        if (k < 0 || id < 0) return;
        const d3 vv = seg_vel64(f4pi, ld3(pos, id), ld3(pos, links[id].x), ld3(pos, k));
        acc[v][0] += vv.x;
        acc[v][1] += vv.y;
        acc[v][2] += vv.z;
      }
    };
    auto stage_one = [&](int m) -> SrcVals {
      if (m >= s1 || status[m].x == OV_EMPTY) return src_none();
      const int f = links[m].x;
      if (f < 0) return src_none();
      const d3 a = ld3(pos, m), bb = ld3(pos, f);
      const double dx = bb.x - a.x, dy = bb.y - a.y, dz = bb.z - a.z;
      const double far2 = fmax(16.0 * (dx * dx + dy * dy + dz * dz), near2);
      return src_from(a.x - O.x, a.y - O.y, a.z - O.z, dx, dy, dz, far2, m);
    };
    for (int base = s0; base < s1; base += TS) {
      __syncthreads();
      for (int q = threadIdx.x; q < TS / 2; q += TB)
        stage_pair(sh[q], stage_one(base + 2 * q), stage_one(base + 2 * q + 1));
      __syncthreads();
      const int nrec = (min(TS, s1 - base) + 1) / 2;   // records holding a source
      for (int q0 = 0; q0 < nrec; q0 += 16) {
        f2 bsum[kTT][3];
#pragma unroll
        for (int k = 0; k < kTT; ++k) bsum[k][0] = bsum[k][1] = bsum[k][2] = f2_splat(0.f);
        const int q1 = min(q0 + 16, nrec);
#pragma unroll 2
        for (int q = q0; q < q1; ++q) pair_interact<kTwo>(sh[q], T, bsum, special);
#pragma unroll
        for (int k = 0; k < kTT; ++k) {
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            float lo, hi;
            f2_unpack(bsum[k][c], lo, hi);
            acc[k][c] += f4pi * ((double)lo + (double)hi);
          }
        }
      }
    }
#pragma unroll
    for (int u = 0; u < kTT; ++u) {
      const int k = w.y + threadIdx.x + TB * u;
      if (k < s1) out(P, k, kk[u] >= 0, mk3(acc[u][0], acc[u][1], acc[u][2]));
    }
  }
}

// Mixed form in chain order (chain_sweep, ov_pair.cuh): each system's
// segments in slot order, where its rings run slot after slot, so a chained
// segment shares its end node with the next and each node's offset and
// 1/|R| serve both; a ring's closing segment takes the two-source form.
// Two-float offsets from the coordinate origin (the systems span whole
// rings, and a slot may be EMPTY); near pairs and pairs at the colinearity
// cut-off in FP64, FP32 partial sums over 32 segments added into FP64 sums.
template <int TB>
__global__ void __launch_bounds__(TB) k_batch_bs_chain(OvParams P, BatchView B,
                                                       const double* __restrict__ pos,
                                                       const int2* __restrict__ links,
                                                       const int2* __restrict__ status,
                                                       StoreSums out, int* __restrict__ work) {
  __shared__ ChainNode<true> sh_node[kCH + 1];
  __shared__ ChainSeg sh_seg[kCH];
  __shared__ PairSrc<true> sh_irr[kCH];
  __shared__ int sh_irr_id[2 * kCH];
  __shared__ int sh_item, sh_n_irr;
  const double f4pi = P.f4pi;
  const d3 O = mk3(0, 0, 0);
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) sh_item = atomicAdd(work, 1);
    __syncthreads();
    const int it = sh_item;
    if (it >= B.n_items) return;
    const int2 w = B.items[it];
    const int s0 = B.off[w.x], s1 = B.off[w.x + 1];
    const double near2 = B.near2[w.x];
    int kk[kTT];
    PairTargets T;
    double acc[kTT][3];
#pragma unroll
    for (int u = 0; u < kTT; ++u) {
      const int k = w.y + threadIdx.x + TB * u;
      const bool act = k < s1 && status[k].x == OV_FREE;
      kk[u] = act ? k : -1;
      const d3 r = act ? ld3(pos, k) : O;
      set_target(T, u, r.x, r.y, r.z);
      acc[u][0] = acc[u][1] = acc[u][2] = 0;
    }
    auto special = [&](int u, int id) {
#pragma unroll
      for (int v = 0; v < kTT; ++v) {
        if (v != u) continue;
        const int k = kk[v];
        if (k < 0 || id < 0) return;
        const d3 vv = seg_vel64(f4pi, ld3(pos, id), ld3(pos, links[id].x), ld3(pos, k));
        acc[v][0] += vv.x;
        acc[v][1] += vv.y;
        acc[v][2] += vv.z;
      }
    };
    // the segment starting at slot m: forward slot (or -1), vector, far radius
    auto seg_of = [&](int m, double* d, double* far2) -> int {
      if (m >= s1 || status[m].x == OV_EMPTY) return -1;
      const int f = links[m].x;
      if (f < 0) return -1;
      const d3 a = ld3(pos, m), bb = ld3(pos, f);
      d[0] = bb.x - a.x;
      d[1] = bb.y - a.y;
      d[2] = bb.z - a.z;
      *far2 = fmax(16.0 * (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]), near2);
      return f;
    };
    for (int sb = s0; sb < s1; sb += 2 * kCH) {
      __syncthreads();
      if (threadIdx.x == 0) sh_n_irr = 0;
      __syncthreads();
      for (int i = threadIdx.x; i <= kCH; i += TB) {
        double off[2][3];
        bool valid[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int m = sb + i + h * kCH;
          valid[h] = m < s1 && status[m].x != OV_EMPTY;
          const d3 p = valid[h] ? ld3(pos, m) : O;
          off[h][0] = p.x;
          off[h][1] = p.y;
          off[h][2] = p.z;
        }
        chain_node_set<true>(sh_node[i], off, valid);
      }
      for (int i = threadIdx.x; i < kCH; i += TB) {
        float dd[2][3], f2v[2];
        int idv[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int m = sb + i + h * kCH;
          double d[3], far2 = 0;
          const int f = seg_of(m, d, &far2);
          dd[h][0] = dd[h][1] = dd[h][2] = 0.f;
          f2v[h] = 0.f;
          idv[h] = -1;
          if (f < 0) continue;
          if (f != m + 1) {
            sh_irr_id[atomicAdd(&sh_n_irr, 1)] = m;
            continue;
          }
          dd[h][0] = (float)d[0];
          dd[h][1] = (float)d[1];
          dd[h][2] = (float)d[2];
          f2v[h] = (float)far2;
          idv[h] = m;
        }
        chain_seg_set(sh_seg[i], dd, f2v, idv);
      }
      __syncthreads();
      const int n_irr = sh_n_irr;
      auto stage_slot = [&](int m) -> SrcVals {
        double d[3], far2 = 0;
        if (m < 0 || seg_of(m, d, &far2) < 0) return src_none();
        const d3 a = ld3(pos, m);
        return src_from(a.x, a.y, a.z, d[0], d[1], d[2], far2, m);
      };
      for (int q = threadIdx.x; 2 * q < n_irr; q += TB)
        stage_pair(sh_irr[q], stage_slot(sh_irr_id[2 * q]),
                   stage_slot(2 * q + 1 < n_irr ? sh_irr_id[2 * q + 1] : -1));
      __syncthreads();
      chain_sweep<true>(sh_node, sh_seg, T, acc, f4pi, special);
      f2 b[kTT][3];
#pragma unroll
      for (int u = 0; u < kTT; ++u) b[u][0] = b[u][1] = b[u][2] = f2_splat(0.f);
      for (int q = 0; 2 * q < n_irr; ++q) pair_interact<true>(sh_irr[q], T, b, special);
#pragma unroll
      for (int u = 0; u < kTT; ++u) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          float lo, hi;
          f2_unpack(b[u][c], lo, hi);
          acc[u][c] += f4pi * ((double)lo + (double)hi);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < kTT; ++u) {
      const int k = w.y + threadIdx.x + TB * u;
      if (k < s1) out(P, k, kk[u] >= 0, mk3(acc[u][0], acc[u][1], acc[u][2]));
    }
  }
}

// per system: near2 = (factor * longest segment)^2
__global__ void k_sys_near2(const int* __restrict__ off, const double* __restrict__ pos,
                            const int2* __restrict__ links, const int2* __restrict__ status,
                            double factor, int n_sys, double* near2) {
  __shared__ double sh[32];
  for (int s = blockIdx.x; s < n_sys; s += gridDim.x) {
    double mx = 0;
    for (int m = off[s] + threadIdx.x; m < off[s + 1]; m += blockDim.x) {
      if (status[m].x == OV_EMPTY) continue;
      const int f = links[m].x;
      if (f < 0) continue;
      const d3 d = ld3(pos, f) - ld3(pos, m);
      mx = fmax(mx, dot3(d, d));
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
      double b = 0;
      for (int i = 0; i < (int)(blockDim.x >> 5); ++i) b = fmax(b, sh[i]);
      near2[s] = factor * factor * b;
    }
  }
}

__global__ void k_advance_time(double* t, double dt) { t[0] += dt; }

using BsKernel = void (*)(OvParams, BatchView, const double*, const int2*, const int2*, StoreSums, int*);

// the kernel shapes the autotuner chooses from
struct Shape {
  int tb, ts;
  BsKernel k64, kmixed;
};
#define OV_SHAPE(TB, TS) {TB, TS, k_batch_bs64<TB, TS>, k_batch_bs_mixed<TB, TS>}
// sources_per_tile 0: the mixed form in chain order (tiles of 128 segments);
// the FP64 form as with 128
#define OV_SHAPE_CHAIN(TB) {TB, 0, k_batch_bs64<TB, 128>, k_batch_bs_chain<TB>}
const Shape kShapes[] = {
    OV_SHAPE(64, 64),  OV_SHAPE(64, 128),  OV_SHAPE(64, 256),  OV_SHAPE(128, 64), OV_SHAPE(128, 128),
    OV_SHAPE(128, 256), OV_SHAPE(256, 64), OV_SHAPE(256, 128), OV_SHAPE(256, 256), OV_SHAPE_CHAIN(64),
    OV_SHAPE_CHAIN(128), OV_SHAPE_CHAIN(256),
};
#undef OV_SHAPE
#undef OV_SHAPE_CHAIN
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);

int find_shape(int tb, int ts) {
  for (int i = 0; i < kNumShapes; ++i)
    if (kShapes[i].tb == tb && kShapes[i].ts == ts) return i;
  return -1;
}

}  // namespace

bool ov_capture_params(const tangle_state* t, OvParams& P);

struct ov_batch {
  ov_state_impl s;
  tangle_state hdr;        // box of the ensemble (no node arrays)
  int n_sys = 0;
  std::vector<int> off;    // host copy of the offsets
  std::vector<int> order;  // systems by decreasing slot count
  DevBuf d_off, d_items, d_near2, d_work, d_time;
  int items_tb = 0, n_items = 0;
  int shape = 4;           // kShapes index (128 targets, 128 sources)
  int blocks_per_sm = 0;
  double tuned_ms = 0;
  double n_targets = 0, n_segments = 0, inter_per_eval = 0;
  double evals = 0, interactions = 0, last_run_ms = 0, bs_ms = 0, kernels_per_step = 0;
  cudaEvent_t ev_bs[8] = {};
  cudaEvent_t ev_run0 = nullptr, ev_run1 = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

bool build_items(ov_batch* b, int tb) {
  if (b->items_tb == tb) return true;
  std::vector<int2> items;
  for (int s : b->order)
    for (int t0 = b->off[s]; t0 < b->off[s + 1]; t0 += tb) items.push_back(make_int2(s, t0));
  b->n_items = (int)items.size();
  if (!b->d_items.reserve(sizeof(int2) * std::max<size_t>(1, items.size()))) return false;
  if (!items.empty())
    OV_TRY_CUDA(cudaMemcpy(b->d_items.p, items.data(), sizeof(int2) * items.size(),
                           cudaMemcpyHostToDevice));
  b->items_tb = tb;
  return true;
}

// SMs x resident blocks per SM of each kernel shape and form, looked up on
// first use (before any graph capture: ov_batch_run calls it first)
int g_sms = 0;
int g_occ[kNumShapes][2] = {};

bool prepare_shape(int shape, bool mixed) {
  if (!g_sms) {
    int dev = 0;
    OV_TRY_CUDA(cudaGetDevice(&dev));
    OV_TRY_CUDA(cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev));
    if (g_sms <= 0) g_sms = 1;
  }
  int& occ = g_occ[shape][mixed ? 1 : 0];
  const Shape& sh = kShapes[shape];
  if (!occ) {
    OV_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, mixed ? sh.kmixed : sh.k64, sh.tb, 0));
    if (occ < 1) occ = 1;
  }
  return true;
}

int grid_for(const ov_batch* b, bool mixed) {
  int per_sm = g_occ[b->shape][mixed ? 1 : 0];
  if (per_sm < 1) per_sm = 1;
  if (b->blocks_per_sm > 0) per_sm = std::min(per_sm, b->blocks_per_sm);
  return std::max(1, std::min(b->n_items, g_sms * per_sm));
}

// the Biot-Savart sum of every system at positions pos -> v_nl; work: a
// zeroed counter
// targets per work item of a kernel shape and form
int item_targets(int shape, bool mixed) { return kShapes[shape].tb * (mixed ? kTT : 1); }

bool launch_bs(ov_batch* b, const double* pos, double* v_nl, int* work) {
  const Shape& sh = kShapes[b->shape];
  const bool mixed = b->s.P.precision == OV_PREC_MIXED;
  if (!build_items(b, item_targets(b->shape, mixed))) return false;
  if (b->n_items == 0) return true;
  BatchView B{b->d_off.as<int>(), b->d_items.as<int2>(), b->d_near2.as<double>(), b->n_items};
  BsKernel k = mixed ? sh.kmixed : sh.k64;
  if (!g_occ[b->shape][mixed ? 1 : 0] && !prepare_shape(b->shape, mixed)) return false;
  const int grid = grid_for(b, mixed);
  k<<<grid, sh.tb, 0, b->s.stream>>>(b->s.P, B, pos, b->s.links.as<int2>(), b->s.status.as<int2>(),
                                     StoreSums{v_nl}, work);
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  return true;
}

bool launch_near2(ov_batch* b, const double* pos) {
  if (b->s.P.precision != OV_PREC_MIXED || b->n_sys == 0) return true;
  const int grid = std::min(b->n_sys, 4096);
  k_sys_near2<<<grid, 128, 0, b->s.stream>>>(b->d_off.as<int>(), pos, b->s.links.as<int2>(),
                                             b->s.status.as<int2>(), ov_get_mixed_near_factor(),
                                             b->n_sys, b->d_near2.as<double>());
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  return true;
}

// geometry + Biot-Savart + epilogue at positions pos (time t0 + *t_dev)
bool enqueue_eval(ov_batch* b, const double* pos, double* dxi, double* tan, double* nrm, double* vels,
                  double* vs, const double* t_dev, double t0, int* work, cudaEvent_t e0, cudaEvent_t e1) {
  ov_state_impl* s = &b->s;
  int* flag = s->dflag.as<int>();
  if (!ov_launch_geometry(s->stream, s->P, s->links.as<int2>(), s->status.as<int2>(), pos, dxi, tan, nrm,
                          s->n, flag))
    return false;
  if (!s->P.lia_only) {
    if (e0) OV_TRY_CUDA(cudaEventRecord(e0, s->stream));
    if (!launch_bs(b, pos, s->v_nl.as<double>(), work)) return false;
    if (e1) OV_TRY_CUDA(cudaEventRecord(e1, s->stream));
  }
  return ov_launch_epilogue(s->stream, s->P, s->links.as<int2>(), s->status.as<int2>(), t_dev, t0, pos,
                            tan, nrm, s->v_nl.as<double>(), nullptr, vels, vs, 0, s->n, flag);
}

// one RK4 step (update_tangle + rk4_step2, src/vortex_dynamics.c:58-117) at
// time *t_dev, which it then advances by dt.  Per stage: the geometry
// kernels, the persistent Biot-Savart kernel, the epilogue and the stage
// update.  (One kernel for the whole stage, with each target's geometry,
// epilogue and update after its sums, measured 74.7 ms per step against
// 52 ms: the FP64 per-node work ran at the sum kernel's occupancy.)
bool enqueue_step(ov_batch* b, double dt, bool classic) {
  ov_state_impl* s = &b->s;
  const int2* st = s->status.as<int2>();
  double* x0 = s->pos.as<double>();
  double* xs = s->spos.as<double>();
  double* ks[3] = {s->k2.as<double>(), s->k3.as<double>(), s->k4.as<double>()};
  const double h[3] = {dt / 2, dt / 2, classic ? dt : dt / 2};
  const double toff[3] = {dt / 2, dt / 2, dt};
  const double* t_dev = b->d_time.as<double>();
  int* work = b->d_work.as<int>();
  OV_TRY_CUDA(cudaMemsetAsync(work, 0, 4 * sizeof(int), s->stream));
  if (!launch_near2(b, x0)) return false;
  if (!enqueue_eval(b, x0, s->dxi.as<double>(), s->tan.as<double>(), s->nrm.as<double>(),
                    s->vels.as<double>(), s->vs.as<double>(), t_dev, 0.0, work, nullptr, nullptr))
    return false;
  for (int q = 0; q < 3; ++q) {
    const double* prev = q == 0 ? s->vels.as<double>() : ks[q - 1];
    if (!ov_launch_euler(s->stream, st, x0, prev, h[q], xs, s->n)) return false;
    if (!enqueue_eval(b, xs, s->sdxi.as<double>(), s->stan.as<double>(), s->snrm.as<double>(), ks[q],
                      s->svs.as<double>(), t_dev, toff[q], work + q + 1, nullptr, nullptr))
      return false;
  }
  if (!ov_launch_rk4_combine(s->stream, st, s->vels.as<double>(), ks[0], ks[1], ks[2], dt, x0, s->n))
    return false;
  k_advance_time<<<1, 1, 0, s->stream>>>(b->d_time.as<double>(), dt);
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  return true;
}

// one Biot-Savart launch at the current positions, timed with events
bool time_bs(ov_batch* b, double* ms_out) {
  ov_state_impl* s = &b->s;
  if (!launch_near2(b, s->pos.as<double>())) return false;
  OV_TRY_CUDA(cudaMemsetAsync(b->d_work.p, 0, sizeof(int), s->stream));
  OV_TRY_CUDA(cudaEventRecord(b->ev_bs[0], s->stream));
  if (!launch_bs(b, s->pos.as<double>(), s->v_nl.as<double>(), b->d_work.as<int>())) return false;
  OV_TRY_CUDA(cudaEventRecord(b->ev_bs[1], s->stream));
  OV_TRY_CUDA(cudaStreamSynchronize(s->stream));
  float ms = 0;
  OV_TRY_CUDA(cudaEventElapsedTime(&ms, b->ev_bs[0], b->ev_bs[1]));
  *ms_out = ms;
  return true;
}

bool read_flag(ov_batch* b, const char* where) {
  int h = 0;
  OV_TRY_CUDA(cudaMemcpyAsync(&h, b->s.dflag.p, sizeof(int), cudaMemcpyDeviceToHost, b->s.stream));
  OV_TRY_CUDA(cudaStreamSynchronize(b->s.stream));
  return ov_flag_status(h, where);
}

bool refresh_params(ov_batch* b) {
  if (!ov_capture_params(&b->hdr, b->s.P)) return false;
  b->s.P.n_img = 0;
  return true;
}

void drop_graph(ov_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;
}

}  // namespace

extern "C" {

ov_batch* ov_batch_create(const struct tangle_state* all, int n_systems, const int* offsets) {
  ov_clear_error();
  if (!all || !offsets || n_systems < 1 || all->N < 0) {
    ov_set_error(OV_ERR_INVALID, "ov_batch_create: null tangle/offsets or %d systems", n_systems);
    return nullptr;
  }
  if (offsets[0] != 0 || offsets[n_systems] != all->N) {
    ov_set_error(OV_ERR_INVALID, "ov_batch_create: offsets must run from 0 to N = %d", all->N);
    return nullptr;
  }
  for (int s = 0; s < n_systems; ++s)
    if (offsets[s + 1] < offsets[s]) {
      ov_set_error(OV_ERR_INVALID, "ov_batch_create: offsets decrease at system %d", s);
      return nullptr;
    }
  for (int w = 0; w < 6; ++w)
    if (all->box.wall[w] != WALL_OPEN) {
      ov_set_error(OV_ERR_INVALID, "ov_batch_create: batched systems need open boundaries (wall %d)", w);
      return nullptr;
    }
  if (all->bimg.n != 0) {
    ov_set_error(OV_ERR_INVALID, "ov_batch_create: batched systems take no boundary images");
    return nullptr;
  }
  if (all->N > 0 && (!all->status || !all->connections || !all->vnodes)) {
    ov_set_error(OV_ERR_INVALID, "ov_batch_create: tangle without node arrays");
    return nullptr;
  }
  double nt = 0, ns = 0, inter = 0;
  for (int s = 0; s < n_systems; ++s) {
    double t_s = 0, g_s = 0;
    for (int k = offsets[s]; k < offsets[s + 1]; ++k) {
      const int st = all->status[k].status;
      if (st == EMPTY) continue;
      if (st != FREE) {
        ov_set_error(OV_ERR_INVALID, "ov_batch_create: node %d has status %d (free or empty only)", k, st);
        return nullptr;
      }
      const int f = all->connections[k].forward, r = all->connections[k].reverse;
      if ((f >= 0 && (f < offsets[s] || f >= offsets[s + 1])) ||
          (r >= 0 && (r < offsets[s] || r >= offsets[s + 1]))) {
        ov_set_error(OV_ERR_INVALID, "ov_batch_create: node %d links outside system %d", k, s);
        return nullptr;
      }
      t_s += 1;
      if (f >= 0) g_s += 1;
    }
    nt += t_s;
    ns += g_s;
    inter += t_s * g_s;
  }
  ov_batch* b = new ov_batch();
  b->hdr = *all;
  b->hdr.N = 0;
  b->hdr.vnodes = nullptr;
  b->n_sys = n_systems;
  b->off.assign(offsets, offsets + n_systems + 1);
  b->order.resize(n_systems);
  for (int s = 0; s < n_systems; ++s) b->order[s] = s;
  std::stable_sort(b->order.begin(), b->order.end(), [&](int x, int y) {
    return b->off[x + 1] - b->off[x] > b->off[y + 1] - b->off[y];
  });
  b->n_targets = nt;
  b->n_segments = ns;
  b->inter_per_eval = inter;
  bool ok = ov_upload_tangle(&b->s, all) && refresh_params(b) &&
            b->d_off.reserve(sizeof(int) * (n_systems + 1)) &&
            b->d_near2.reserve(sizeof(double) * n_systems) && b->d_work.reserve(64) &&
            b->d_time.reserve(64);
  if (ok) {
    ok = ov_cuda_ok(cudaMemcpyAsync(b->d_off.p, offsets, sizeof(int) * (n_systems + 1),
                                    cudaMemcpyHostToDevice, b->s.stream),
                    "cudaMemcpyAsync") &&
         ov_cuda_ok(cudaMemsetAsync(b->d_near2.p, 0, sizeof(double) * n_systems, b->s.stream),
                    "cudaMemsetAsync") &&
         ov_cuda_ok(cudaMemsetAsync(b->d_time.p, 0, 64, b->s.stream), "cudaMemsetAsync");
    for (int i = 0; ok && i < 8; ++i) ok = ov_cuda_ok(cudaEventCreate(&b->ev_bs[i]), "cudaEventCreate");
    ok = ok && ov_cuda_ok(cudaEventCreate(&b->ev_run0), "cudaEventCreate") &&
         ov_cuda_ok(cudaEventCreate(&b->ev_run1), "cudaEventCreate");
    // stage positions of EMPTY slots are never written: keep them defined
    if (ok && all->N > 0)
      ok = ov_cuda_ok(cudaMemcpyAsync(b->s.spos.p, b->s.pos.p, sizeof(double) * 3 * all->N,
                                      cudaMemcpyDeviceToDevice, b->s.stream),
                      "cudaMemcpyAsync");
    ok = ok && ov_cuda_ok(cudaStreamSynchronize(b->s.stream), "cudaStreamSynchronize");
  }
  if (!ok) {
    int e = ov_last_error();
    ov_batch_destroy(b);
    if (!ov_last_error()) ov_set_error(e ? e : OV_ERR_CUDA, "ov_batch_create failed");
    return nullptr;
  }
  return b;
}

void ov_batch_destroy(ov_batch* b) {
  if (!b) return;
  drop_graph(b);
  for (cudaEvent_t& e : b->ev_bs)
    if (e) cudaEventDestroy(e);
  if (b->ev_run0) cudaEventDestroy(b->ev_run0);
  if (b->ev_run1) cudaEventDestroy(b->ev_run1);
  DevBuf* bufs[] = {&b->d_off, &b->d_items, &b->d_near2, &b->d_work, &b->d_time};
  for (DevBuf* d : bufs) d->release();
  DevBuf* sb[] = {&b->s.pos, &b->s.links, &b->s.status, &b->s.dxi, &b->s.tan, &b->s.nrm, &b->s.vels,
                  &b->s.vs, &b->s.pos0, &b->s.spos, &b->s.sdxi, &b->s.stan, &b->s.snrm, &b->s.svs,
                  &b->s.k2, &b->s.k3, &b->s.k4, &b->s.v_nl, &b->s.v_img, &b->s.dflag};
  for (DevBuf* d : sb) d->release();
  if (b->s.stream) cudaStreamDestroy(b->s.stream);
  if (b->s.ev0) cudaEventDestroy(b->s.ev0);
  if (b->s.ev1) cudaEventDestroy(b->s.ev1);
  if (b->s.ev2) cudaEventDestroy(b->s.ev2);
  delete b;
}

int ov_batch_update(ov_batch* b, double t) {
  ov_clear_error();
  if (!b) { ov_set_error(OV_ERR_INVALID, "null batch"); return ov_last_error(); }
  if (!refresh_params(b)) return ov_last_error();
  ov_state_impl* s = &b->s;
  bool ok = ov_cuda_ok(cudaMemsetAsync(s->dflag.p, 0, sizeof(int), s->stream), "cudaMemsetAsync") &&
            ov_cuda_ok(cudaMemsetAsync(b->d_work.p, 0, sizeof(int), s->stream), "cudaMemsetAsync") &&
            launch_near2(b, s->pos.as<double>()) &&
            enqueue_eval(b, s->pos.as<double>(), s->dxi.as<double>(), s->tan.as<double>(),
                         s->nrm.as<double>(), s->vels.as<double>(), s->vs.as<double>(), nullptr, t,
                         b->d_work.as<int>(), b->ev_bs[0], b->ev_bs[1]) &&
            read_flag(b, "ov_batch_update");
  if (!ok) return ov_last_error();
  float ms = 0;
  if (!s->P.lia_only && !ov_cuda_ok(cudaEventElapsedTime(&ms, b->ev_bs[0], b->ev_bs[1]),
                                    "cudaEventElapsedTime"))
    return ov_last_error();
  b->bs_ms = ms;
  b->evals += 1;
  b->interactions += s->P.lia_only ? 0 : b->inter_per_eval;
  return OV_OK;
}

int ov_batch_run(ov_batch* b, double t0, double dt, int nsteps) {
  ov_clear_error();
  if (!b || nsteps < 0) { ov_set_error(OV_ERR_INVALID, "null batch or negative step count"); return ov_last_error(); }
  if (!refresh_params(b)) return ov_last_error();
  ov_state_impl* s = &b->s;
  const bool classic = ov_get_rk4_classic() != 0;
  // one RK4 step as a graph (the parameters, the kernel shape and dt are
  // baked in, so it is captured again on every call)
  drop_graph(b);
  if (!build_items(b, item_targets(b->shape, s->P.precision == OV_PREC_MIXED)) ||
      !prepare_shape(b->shape, s->P.precision == OV_PREC_MIXED))
    return ov_last_error();
  const long long before = ov_launches();
  cudaGraph_t graph = nullptr;
  if (!ov_cuda_ok(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal),
                  "cudaStreamBeginCapture"))
    return ov_last_error();
  const bool enq = enqueue_step(b, dt, classic);
  const cudaError_t ce = cudaStreamEndCapture(s->stream, &graph);
  const long long per_step = ov_launches() - before;
  ov_note_launch((int)-per_step);   // counted again per replay below
  if (!enq || !ov_cuda_ok(ce, "cudaStreamEndCapture")) {
    if (graph) cudaGraphDestroy(graph);
    return ov_last_error() ? ov_last_error() : OV_ERR_CUDA;
  }
  const bool inst = ov_cuda_ok(cudaGraphInstantiate(&b->exec, graph, 0), "cudaGraphInstantiate");
  cudaGraphDestroy(graph);
  if (!inst) return ov_last_error();
  b->kernels_per_step = (double)per_step;
  bool ok = ov_cuda_ok(cudaMemcpyAsync(b->d_time.p, &t0, sizeof(double), cudaMemcpyHostToDevice,
                                       s->stream),
                       "cudaMemcpyAsync") &&
            ov_cuda_ok(cudaMemsetAsync(s->dflag.p, 0, sizeof(int), s->stream), "cudaMemsetAsync") &&
            ov_cuda_ok(cudaEventRecord(b->ev_run0, s->stream), "cudaEventRecord");
  for (int i = 0; ok && i < nsteps; ++i) {
    ok = ov_cuda_ok(cudaGraphLaunch(b->exec, s->stream), "cudaGraphLaunch");
    if (ok) ov_note_launch((int)per_step);
  }
  ok = ok && ov_cuda_ok(cudaEventRecord(b->ev_run1, s->stream), "cudaEventRecord") &&
       read_flag(b, "ov_batch_run");
  if (!ok) return ov_last_error();
  float ms = 0;
  if (!ov_cuda_ok(cudaEventElapsedTime(&ms, b->ev_run0, b->ev_run1), "cudaEventElapsedTime"))
    return ov_last_error();
  b->last_run_ms = ms;
  // device time of one Biot-Savart launch at the final positions, outside
  // the graph (its result lands in scratch only)
  if (nsteps > 0 && !s->P.lia_only && !time_bs(b, &b->bs_ms)) return ov_last_error();
  b->evals += 4.0 * nsteps;
  b->interactions += s->P.lia_only ? 0 : 4.0 * nsteps * b->inter_per_eval;
  return OV_OK;
}

int ov_batch_download(ov_batch* b, struct tangle_state* all, int what) {
  ov_clear_error();
  if (!b || !all) { ov_set_error(OV_ERR_INVALID, "null batch or tangle"); return ov_last_error(); }
  if (!ov_download_fields(&b->s, all, what)) return ov_last_error();
  return OV_OK;
}

int ov_batch_set_tuning(ov_batch* b, const ov_batch_tuning* t) {
  ov_clear_error();
  if (!b || !t) { ov_set_error(OV_ERR_INVALID, "null batch or tuning"); return ov_last_error(); }
  const int i = find_shape(t->targets_per_block, t->sources_per_tile);
  if (i < 0 || t->blocks_per_sm < 0) {
    ov_set_error(OV_ERR_INVALID, "ov_batch_set_tuning: no kernel shape %d targets x %d sources",
                 t->targets_per_block, t->sources_per_tile);
    return ov_last_error();
  }
  b->shape = i;
  b->blocks_per_sm = t->blocks_per_sm;
  drop_graph(b);
  return OV_OK;
}

int ov_batch_get_tuning(ov_batch* b, ov_batch_tuning* out) {
  if (!b || !out) return OV_ERR_INVALID;
  out->targets_per_block = kShapes[b->shape].tb;
  out->sources_per_tile = kShapes[b->shape].ts;
  out->blocks_per_sm = b->blocks_per_sm;
  out->kernel_ms = b->tuned_ms;
  return OV_OK;
}

// Times every kernel shape (one warm-up and two timed launches each, at the
// current positions and precision) and keeps the fastest.
int ov_batch_autotune(ov_batch* b, ov_batch_tuning* out) {
  ov_clear_error();
  if (!b) { ov_set_error(OV_ERR_INVALID, "null batch"); return ov_last_error(); }
  if (!refresh_params(b)) return ov_last_error();
  ov_state_impl* s = &b->s;
  if (!launch_near2(b, s->pos.as<double>())) return ov_last_error();
  const int keep_bps = b->blocks_per_sm;
  int best = -1, best_bps = 0;
  float best_ms = 0;
  const int bps_opts[2] = {0, 2};
  for (int i = 0; i < kNumShapes; ++i) {
    for (int bo : bps_opts) {
      b->shape = i;
      b->blocks_per_sm = bo;
      float tot = 0;
      bool ok = true;
      for (int rep = 0; ok && rep < 3; ++rep) {
        ok = ov_cuda_ok(cudaMemsetAsync(b->d_work.p, 0, sizeof(int), s->stream), "cudaMemsetAsync") &&
             ov_cuda_ok(cudaEventRecord(b->ev_bs[0], s->stream), "cudaEventRecord") &&
             launch_bs(b, s->pos.as<double>(), s->v_nl.as<double>(), b->d_work.as<int>()) &&
             ov_cuda_ok(cudaEventRecord(b->ev_bs[1], s->stream), "cudaEventRecord") &&
             ov_cuda_ok(cudaStreamSynchronize(s->stream), "cudaStreamSynchronize");
        float ms = 0;
        ok = ok && ov_cuda_ok(cudaEventElapsedTime(&ms, b->ev_bs[0], b->ev_bs[1]), "cudaEventElapsedTime");
        if (rep > 0) tot += ms;
      }
      if (!ok) {
        b->blocks_per_sm = keep_bps;
        return ov_last_error();
      }
      const float ms = tot / 2;
      if (best < 0 || ms < best_ms) {
        best = i;
        best_bps = bo;
        best_ms = ms;
      }
    }
  }
  b->shape = best;
  b->blocks_per_sm = best_bps;
  b->tuned_ms = best_ms;
  drop_graph(b);
  if (out) ov_batch_get_tuning(b, out);
  return OV_OK;
}

int ov_batch_get_stats(ov_batch* b, ov_batch_stats* out) {
  if (!b || !out) return OV_ERR_INVALID;
  out->evals = b->evals;
  out->interactions = b->interactions;
  out->last_run_ms = b->last_run_ms;
  out->bs_kernel_ms = b->bs_ms;
  out->kernels_per_step = b->kernels_per_step;
  out->n_targets = b->n_targets;
  out->n_segments = b->n_segments;
  out->n_systems = b->n_sys;
  return OV_OK;
}

}  // extern "C"
