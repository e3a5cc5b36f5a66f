// ov_direct.cu - direct (all-pairs) Biot-Savart sums with boundary images.
//
// Replaces the O(N) segment loop of update_velocity (src/tangle.c:611-619)
// run for every node, and the image loop (src/tangle.c:627-636) that repeats
// it at each shifted target: O(N^2 (1 + images)) interactions.
//
// Layout: block = 128 targets x one image (grid.y); source segments are
// staged in shared memory 128 at a time and every thread sweeps the tile for
// its own target.  Per-image partial sums land in img_part[j][k] and are
// summed in image-table order so the result is deterministic.
//
// FP64 form: the reference's formula with refined reciprocal square roots and
// reciprocals instead of IEEE square roots and divisions, and its cut-offs
// decided by its own operations (seg_vel64_nr).
// Mixed form (k_direct_mixed_pairs): sources staged two by two as FP32
// offsets from the block's first target (the subtraction done in FP64,
// rounded once) and evaluated two per f32x2 instruction (ov_pair.cuh); near
// or borderline-colinear pairs fall back to seg_vel64 from the FP64 table;
// sums accumulate in FP64.
#include <stdlib.h>

#include <algorithm>

#include "ov_internal.h"
#include "ov_pair.cuh"

namespace {

constexpr int kTB = 128;   // targets per block
constexpr int kTS = 128;   // sources per shared-memory tile

struct SegTab {
  const double* r1r2;   // 6 doubles per source slot: r1, wrapped r2
  const int* fwd;       // forward slot per source slot (-1: no segment)
};

// r1 and the wrapped r2 of each slot's forward segment
__global__ void k_segtab(OvParams P, const double* __restrict__ pos, const int2* __restrict__ links,
                         const int2* __restrict__ status, double* r1r2, int* fwd, int n) {
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  int f = links[m].x;
  if (status[m].x == OV_EMPTY) f = -1;
  fwd[m] = f;
  d3 a = ld3(pos, m);
  d3 b = f >= 0 ? pwrap(P, a, ld3(pos, f)) : a;
  double* o = r1r2 + 6 * m;
  o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = b.x; o[4] = b.y; o[5] = b.z;
}

// Targets: either node slots (pts == nullptr: slot k, status-filtered) or
// explicit points.  Sources: all slots, or the list `only`; split z of the
// grid takes sources [z chunk, (z + 1) chunk) and writes its own partial
// sums part[z][image][target].
__global__ void __launch_bounds__(kTB) k_direct64(OvParams P, SegTab S, int n_src, const int* only,
                                                  const double* __restrict__ tpos,
                                                  const int2* __restrict__ tstatus,
                                                  const int* __restrict__ tskip, int n_t,
                                                  double* __restrict__ part, int chunk) {
  __shared__ double sh_r[kTS][9];   // r1, wrapped r2, d = r2 - r1
  __shared__ int sh_id[kTS][2];
  const int j = blockIdx.y;  // 0: the tangle itself, j >= 1: image j-1
  const int k = blockIdx.x * kTB + threadIdx.x;
  bool act = k < n_t;
  if (act && tstatus) act = tstatus[k].x != OV_EMPTY && tstatus[k].x != OV_PINNED;
  d3 r = mk3(0, 0, 0);
  int skip = -1;
  if (act) {
    r = ld3(tpos, k);
    if (j > 0) r = image_point(P, j - 1, r);
    else skip = tskip ? tskip[k] : (tstatus ? k : -1);
  }
  double ax = 0, ay = 0, az = 0;
  const double f4pi = P.f4pi;
  const int s_lo = blockIdx.z * chunk, s_hi = min(n_src, s_lo + chunk);
  for (int base = s_lo; base < s_hi; base += kTS) {
    __syncthreads();
    for (int q = threadIdx.x; q < kTS; q += kTB) {
      int m = base + q;
      int id = -1, fw = -1;
      if (m < s_hi) {
        id = only ? only[m] : m;
        fw = S.fwd[id];
        const double* src = S.r1r2 + 6 * id;
#pragma unroll
        for (int c = 0; c < 6; ++c) sh_r[q][c] = src[c];
#pragma unroll
        for (int c = 0; c < 3; ++c) sh_r[q][6 + c] = src[3 + c] - src[c];
      }
      sh_id[q][0] = id;
      sh_id[q][1] = fw;
    }
    __syncthreads();
    if (!act) continue;
    int cnt = min(kTS, s_hi - base);
    for (int q = 0; q < cnt; ++q) {
      int id = sh_id[q][0], fw = sh_id[q][1];
      // skip rule of calculate_vs_shift (src/tangle.c:567-569)
      if (fw == -1 || id == skip || fw == skip) continue;
      d3 v = seg_vel64_nr(f4pi, mk3(sh_r[q][0], sh_r[q][1], sh_r[q][2]),
                          mk3(sh_r[q][3], sh_r[q][4], sh_r[q][5]),
                          mk3(sh_r[q][6], sh_r[q][7], sh_r[q][8]), r);
      ax += v.x; ay += v.y; az += v.z;
    }
  }
  if (k < n_t) {
    double* o = part + ((size_t)blockIdx.z * gridDim.y + j) * 3 * n_t + 3 * (size_t)k;
    o[0] = act ? ax : 0; o[1] = act ? ay : 0; o[2] = act ? az : 0;
  }
}

// Mixed form, two sources per instruction.  Block = kPB threads x kTT
// targets (the tree's key order, so close in space) x one image.  The
// origin O is the block's first target, so a single rounding of the
// offsets costs R a few FP32 ulps of |R| + (the block's extent).  A segment
// wrapped across a periodic face may be the one the skip rule drops for its
// end node; for the tangle itself (image 0) it is always evaluated in FP64,
// where that rule is applied.
//
// Shape measured on the 22.4k-point periodic tangle: 128 threads of 2
// targets, at most 96 registers (5 resident blocks per SM), two records per
// unrolled step.
constexpr int kPB = 128;            // threads per block
constexpr int kPTgt = kPB * kTT;    // targets per block
constexpr int kPSrc = 128;          // sources per shared-memory tile (kPSrc / 2 records)

#ifndef OV_DIRECT_PAIRS_MIN_BLOCKS
#define OV_DIRECT_PAIRS_MIN_BLOCKS 5
#endif
__global__ void __launch_bounds__(kPB, OV_DIRECT_PAIRS_MIN_BLOCKS) k_direct_mixed_pairs(
    OvParams P, SegTab S, int n_src, const double* __restrict__ pos, const int2* __restrict__ tstatus,
    const int* __restrict__ order, int n_t, int stride, double* __restrict__ part, int chunk) {
  __shared__ PairSrc<false> sh[kPSrc / 2];
  const int j = blockIdx.y;   // 0: the tangle itself, j >= 1: image j-1
  const int base = blockIdx.x * kPTgt;
  d3 O = ld3(pos, order[base]);
  if (j > 0) O = image_point(P, j - 1, O);
  int kk[kTT];
  PairTargets T;
#pragma unroll
  for (int u = 0; u < kTT; ++u) {
    const int i = base + threadIdx.x + kPB * u;
    int k = i < n_t ? order[i] : -1;
    if (k >= 0 && (tstatus[k].x == OV_EMPTY || tstatus[k].x == OV_PINNED)) k = -1;
    kk[u] = k;
    d3 r = O;
    if (k >= 0) {
      r = ld3(pos, k);
      if (j > 0) r = image_point(P, j - 1, r);
    }
    set_target(T, u, r.x - O.x, r.y - O.y, r.z - O.z);
  }
  double acc[kTT][3];
#pragma unroll
  for (int u = 0; u < kTT; ++u) acc[u][0] = acc[u][1] = acc[u][2] = 0;
  const double f4pi = P.f4pi;
  // FP64 evaluation of segment id at target u (skip rule of
  // calculate_vs_shift, src/tangle.c:567-569, for the tangle itself)
  auto special = [&](int u, int id) {
#pragma unroll
    for (int v = 0; v < kTT; ++v) {
      if (v != u) continue;
      const int k = kk[v];
      if (k < 0 || id < 0) return;
      const int fw = S.fwd[id];
      if (j == 0 && (id == k || fw == k)) return;
      d3 r = ld3(pos, k);
      if (j > 0) r = image_point(P, j - 1, r);
      const double* sg = S.r1r2 + 6 * (size_t)id;
      const d3 vv = seg_vel64(f4pi, mk3(sg[0], sg[1], sg[2]), mk3(sg[3], sg[4], sg[5]), r);
      acc[v][0] += vv.x;
      acc[v][1] += vv.y;
      acc[v][2] += vv.z;
    }
  };
  const int s_lo = blockIdx.z * chunk, s_hi = min(n_src, s_lo + chunk);
  auto stage_one = [&](int m) -> SrcVals {
    const int id = m < s_hi ? order[m] : -1;
    const int fw = id >= 0 ? S.fwd[id] : -1;
    if (fw < 0) return src_none();
    const double* sg = S.r1r2 + 6 * (size_t)id;
    const double dxx = sg[3] - sg[0], dyy = sg[4] - sg[1], dzz = sg[5] - sg[2];
    double far2 = fmax(16.0 * (dxx * dxx + dyy * dyy + dzz * dzz), P.near2);
    if (j == 0) {
      const d3 e = ld3(pos, fw);
      if (e.x != sg[3] || e.y != sg[4] || e.z != sg[5]) far2 = 1e30;
    }
    return src_from(sg[0] - O.x, sg[1] - O.y, sg[2] - O.z, dxx, dyy, dzz, far2, id);
  };
  for (int sb = s_lo; sb < s_hi; sb += kPSrc) {
    __syncthreads();
    for (int q = threadIdx.x; q < kPSrc / 2; q += kPB)
      stage_pair(sh[q], stage_one(sb + 2 * q), stage_one(sb + 2 * q + 1));
    __syncthreads();
    // FP32 partial sums over 32 sources, each added into the FP64 sums
    for (int q0 = 0; q0 < kPSrc / 2; q0 += 16) {
      f2 b[kTT][3];
#pragma unroll
      for (int k = 0; k < kTT; ++k) b[k][0] = b[k][1] = b[k][2] = f2_splat(0.f);
#pragma unroll 2
      for (int q = q0; q < q0 + 16; ++q) pair_interact<false>(sh[q], T, b, special);
#pragma unroll
      for (int k = 0; k < kTT; ++k) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          float lo, hi;
          f2_unpack(b[k][c], lo, hi);
          acc[k][c] += f4pi * ((double)lo + (double)hi);
        }
      }
    }
  }
#pragma unroll
  for (int u = 0; u < kTT; ++u) {
    const int i = base + threadIdx.x + kPB * u;
    if (i >= n_t) continue;
    double* o = part + ((size_t)blockIdx.z * gridDim.y + j) * 3 * stride + 3 * (size_t)order[i];
    const bool act = kk[u] >= 0;
    o[0] = act ? acc[u][0] : 0;
    o[1] = act ? acc[u][1] : 0;
    o[2] = act ? acc[u][2] : 0;
  }
}

// Mixed form in chain order (k_direct_mixed_chain).  Sources are staged in
// slot order, where a loop's segments follow one another: segment m runs
// from node m to node m + 1 for all but one segment per loop.  Such
// "chained" segments share their end node with the next segment, so each
// node's offset R = r_node - r, |R|^2 and 1/|R| are formed once per target
// and used by both segments that touch it.  Per pair (a = |R|, b = |R'|):
//   u = 1/(ab), den = 1 + R.R' u = 1 + cos, w = u / den
//   v = kappa/4pi (1/a + 1/b) w (R x d)
// R x d, with d the segment vector staged on its own, keeps the FP32 error
// of the cross product at a few ulps of |R||d|.  1 - cos is first estimated
// as 1 - R.R' u, whose error is below 1e-6; only a warp with a pair under
// 2e-6 forms the exact |R x d|^2 u w of the reference's cut-off test.
// That is 24 lane operations and 2 hardware approximations per interaction,
// against 31 and 3 for the two-source form.  Segments that do not chain (a
// loop's closing segment, a segment wrapped across a periodic face, a
// tile's last segment) take the two-source form from a per-tile list.
//
// Tile layout: kCH chained pairs; pair i holds segments sb + i (low half)
// and sb + kCH + i (high half), node pack i holds nodes sb + i and
// sb + kCH + i, for i = 0 .. kCH.
constexpr int kCH = kPSrc / 2;

struct __align__(16) ChainSeg {
  float4 a;      // dx0 dx1 dy0 dy1
  float4 b;      // dz0 dz1 -dx0 -dx1
  float4 c;      // -dy0 -dy1 -dz0 -dz1
  float2 far2;   // FP32 far radius squared per half
  int id[2];     // source slot, -1: contributes nothing
};
template <bool kTwo>
struct __align__(8) ChainNode {
  float2 x, y, z;            // offsets of the two nodes from the block origin
  float2 lx[kTwo ? 1 : 0];   // two-float form: the low parts
  float2 ly[kTwo ? 1 : 0];
  float2 lz[kTwo ? 1 : 0];
};

#ifndef OV_DIRECT_CHAIN_MIN_BLOCKS
#define OV_DIRECT_CHAIN_MIN_BLOCKS 4
#endif
#ifndef OV_DIRECT_CHAIN_UNROLL
#define OV_DIRECT_CHAIN_UNROLL 4
#endif
constexpr int kChainUnroll = OV_DIRECT_CHAIN_UNROLL;
// kTwo: offsets as two floats (hi + lo) for targets and nodes, so R carries
// ~2 ulps of |R| whatever the block's extent: targets may then come in slot
// order (order == nullptr) with no key sort.
template <bool kTwo>
__global__ void __launch_bounds__(kPB, OV_DIRECT_CHAIN_MIN_BLOCKS) k_direct_mixed_chain(
    OvParams P, SegTab S, int n_src, const double* __restrict__ pos, const int2* __restrict__ tstatus,
    const int* __restrict__ order, int n_t, int stride, double* __restrict__ part, int chunk) {
  __shared__ ChainNode<kTwo> sh_node[kCH + 1];
  __shared__ ChainSeg sh_seg[kCH];
  __shared__ PairSrc<kTwo> sh_irr[kPSrc / 2];
  __shared__ int sh_irr_id[kPSrc];
  __shared__ int sh_n_irr;
  const int j = blockIdx.y;   // 0: the tangle itself, j >= 1: image j-1
  const int base = blockIdx.x * kPTgt;
  // origin: the block's first target in key order; in slot order (two-float
  // offsets, where the origin costs no accuracy) the coordinate origin,
  // since a slot there may be EMPTY
  d3 O = order ? ld3(pos, order[base]) : mk3(0, 0, 0);
  if (j > 0) O = image_point(P, j - 1, O);
  int kk[kTT];
  PairTargets T;
#pragma unroll
  for (int u = 0; u < kTT; ++u) {
    const int i = base + threadIdx.x + kPB * u;
    int k = i < n_t ? (order ? order[i] : i) : -1;
    if (k >= 0 && (tstatus[k].x == OV_EMPTY || tstatus[k].x == OV_PINNED)) k = -1;
    kk[u] = k;
    d3 r = O;
    if (k >= 0) {
      r = ld3(pos, k);
      if (j > 0) r = image_point(P, j - 1, r);
    }
    set_target(T, u, r.x - O.x, r.y - O.y, r.z - O.z);
  }
  double acc[kTT][3];
#pragma unroll
  for (int u = 0; u < kTT; ++u) acc[u][0] = acc[u][1] = acc[u][2] = 0;
  const double f4pi = P.f4pi;
  auto special = [&](int u, int id) {
#pragma unroll
    for (int v = 0; v < kTT; ++v) {
      if (v != u) continue;
      const int k = kk[v];
      if (k < 0 || id < 0) return;
      const int fw = S.fwd[id];
      if (j == 0 && (id == k || fw == k)) return;
      d3 r = ld3(pos, k);
      if (j > 0) r = image_point(P, j - 1, r);
      const double* sg = S.r1r2 + 6 * (size_t)id;
      const d3 vv = seg_vel64(f4pi, mk3(sg[0], sg[1], sg[2]), mk3(sg[3], sg[4], sg[5]), r);
      acc[v][0] += vv.x;
      acc[v][1] += vv.y;
      acc[v][2] += vv.z;
    }
  };
  const int s_lo = blockIdx.z * chunk, s_hi = min(n_src, s_lo + chunk);
  // a source by slot for the two-source form (the tangle's own wrapped
  // segments go to FP64, where the skip rule applies)
  auto stage_slot = [&](int id) -> SrcVals {
    const int fw = id >= 0 ? S.fwd[id] : -1;
    if (fw < 0) return src_none();
    const double* sg = S.r1r2 + 6 * (size_t)id;
    const double dxx = sg[3] - sg[0], dyy = sg[4] - sg[1], dzz = sg[5] - sg[2];
    double far2 = fmax(16.0 * (dxx * dxx + dyy * dyy + dzz * dzz), P.near2);
    if (j == 0) {
      const d3 e = ld3(pos, fw);
      if (e.x != sg[3] || e.y != sg[4] || e.z != sg[5]) far2 = 1e30;
    }
    return src_from(sg[0] - O.x, sg[1] - O.y, sg[2] - O.z, dxx, dyy, dzz, far2, id);
  };
  const f2 one = f2_splat(1.0f), two = f2_splat(2.0f);
  for (int sb = s_lo; sb < s_hi; sb += kPSrc) {
    __syncthreads();
    if (threadIdx.x == 0) sh_n_irr = 0;
    __syncthreads();
    // node packs: nodes sb + i and sb + kCH + i (EMPTY or beyond the range:
    // far away, used by no chained segment)
    for (int i = threadIdx.x; i <= kCH; i += kPB) {
      float o[2][3], lo[2][3];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int m = sb + i + h * kCH;
        if (m < n_src && tstatus[m].x != OV_EMPTY) {
          const d3 p = ld3(pos, m);
          const double ox = p.x - O.x, oy = p.y - O.y, oz = p.z - O.z;
          o[h][0] = (float)ox;
          o[h][1] = (float)oy;
          o[h][2] = (float)oz;
          lo[h][0] = (float)(ox - o[h][0]);
          lo[h][1] = (float)(oy - o[h][1]);
          lo[h][2] = (float)(oz - o[h][2]);
        } else {
          o[h][0] = o[h][1] = o[h][2] = 1.0e4f;
          lo[h][0] = lo[h][1] = lo[h][2] = 0.f;
        }
      }
      sh_node[i].x = make_float2(o[0][0], o[1][0]);
      sh_node[i].y = make_float2(o[0][1], o[1][1]);
      sh_node[i].z = make_float2(o[0][2], o[1][2]);
      if constexpr (kTwo) {
        sh_node[i].lx[0] = make_float2(lo[0][0], lo[1][0]);
        sh_node[i].ly[0] = make_float2(lo[0][1], lo[1][1]);
        sh_node[i].lz[0] = make_float2(lo[0][2], lo[1][2]);
      }
    }
    // chained segments; the others to the list
    for (int i = threadIdx.x; i < kCH; i += kPB) {
      float dd[2][3], f2v[2];
      int idv[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int m = sb + i + h * kCH;
        const int fw = m < s_hi ? S.fwd[m] : -1;
        dd[h][0] = dd[h][1] = dd[h][2] = 0.f;
        f2v[h] = 0.f;
        idv[h] = -1;
        if (fw < 0) continue;
        const double* sg = S.r1r2 + 6 * (size_t)m;
        bool chained = fw == m + 1;
        if (chained) {
          const d3 e = ld3(pos, fw);
          chained = e.x == sg[3] && e.y == sg[4] && e.z == sg[5];
        }
        if (!chained) {
          sh_irr_id[atomicAdd(&sh_n_irr, 1)] = m;
          continue;
        }
        const double dxx = sg[3] - sg[0], dyy = sg[4] - sg[1], dzz = sg[5] - sg[2];
        dd[h][0] = (float)dxx;
        dd[h][1] = (float)dyy;
        dd[h][2] = (float)dzz;
        f2v[h] = (float)fmax(16.0 * (dxx * dxx + dyy * dyy + dzz * dzz), P.near2);
        idv[h] = m;
      }
      sh_seg[i].a = make_float4(dd[0][0], dd[1][0], dd[0][1], dd[1][1]);
      sh_seg[i].b = make_float4(dd[0][2], dd[1][2], -dd[0][0], -dd[1][0]);
      sh_seg[i].c = make_float4(-dd[0][1], -dd[1][1], -dd[0][2], -dd[1][2]);
      sh_seg[i].far2 = make_float2(f2v[0], f2v[1]);
      sh_seg[i].id[0] = idv[0];
      sh_seg[i].id[1] = idv[1];
    }
    __syncthreads();
    const int n_irr = sh_n_irr;
    for (int q = threadIdx.x; 2 * q < n_irr; q += kPB)
      stage_pair(sh_irr[q], stage_slot(sh_irr_id[2 * q]), 2 * q + 1 < n_irr ? stage_slot(sh_irr_id[2 * q + 1])
                                                                             : src_none());
    __syncthreads();
    // node 0 of the tile for each target
    f2 Rx[kTT], Ry[kTT], Rz[kTT], R2[kTT], ia[kTT];
    {
      const ChainNode<kTwo> nd = sh_node[0];
      const f2 nx = f2_pack(nd.x.x, nd.x.y), ny = f2_pack(nd.y.x, nd.y.y), nz = f2_pack(nd.z.x, nd.z.y);
#pragma unroll
      for (int u = 0; u < kTT; ++u) {
        Rx[u] = nx - T.x[u];
        Ry[u] = ny - T.y[u];
        Rz[u] = nz - T.z[u];
        if constexpr (kTwo) {
          Rx[u] = Rx[u] + (f2_pack(nd.lx[0].x, nd.lx[0].y) - T.lx[u]);
          Ry[u] = Ry[u] + (f2_pack(nd.ly[0].x, nd.ly[0].y) - T.ly[u]);
          Rz[u] = Rz[u] + (f2_pack(nd.lz[0].x, nd.lz[0].y) - T.lz[u]);
        }
        R2[u] = f2_fma(Rz[u], Rz[u], f2_fma(Ry[u], Ry[u], Rx[u] * Rx[u]));
        ia[u] = f2_rsqrt(R2[u]);
      }
    }
    // FP32 partial sums over 32 segments, each added into the FP64 sums
    for (int i0 = 0; i0 < kCH; i0 += 16) {
      f2 b[kTT][3];
#pragma unroll
      for (int u = 0; u < kTT; ++u) b[u][0] = b[u][1] = b[u][2] = f2_splat(0.f);
#pragma unroll kChainUnroll
      for (int i = i0; i < i0 + 16; ++i) {
        const ChainNode<kTwo> nd = sh_node[i + 1];
        const ChainSeg sg = sh_seg[i];
        const f2 nx = f2_pack(nd.x.x, nd.x.y), ny = f2_pack(nd.y.x, nd.y.y), nz = f2_pack(nd.z.x, nd.z.y);
        f2 nlx, nly, nlz;
        if constexpr (kTwo) {
          nlx = f2_pack(nd.lx[0].x, nd.lx[0].y);
          nly = f2_pack(nd.ly[0].x, nd.ly[0].y);
          nlz = f2_pack(nd.lz[0].x, nd.lz[0].y);
        }
        const f2 dx = f2_pack(sg.a.x, sg.a.y), dy = f2_pack(sg.a.z, sg.a.w), dz = f2_pack(sg.b.x, sg.b.y);
        const f2 ndx = f2_pack(sg.b.z, sg.b.w), ndy = f2_pack(sg.c.x, sg.c.y), ndz = f2_pack(sg.c.z, sg.c.w);
#pragma unroll
        for (int u = 0; u < kTT; ++u) {
          f2 Bx = nx - T.x[u], By = ny - T.y[u], Bz = nz - T.z[u];
          if constexpr (kTwo) {
            Bx = Bx + (nlx - T.lx[u]);
            By = By + (nly - T.ly[u]);
            Bz = Bz + (nlz - T.lz[u]);
          }
          const f2 B2 = f2_fma(Bz, Bz, f2_fma(By, By, Bx * Bx));
          const f2 ib = f2_rsqrt(B2);
          const f2 Cx = f2_fma(Ry[u], dz, Rz[u] * ndy);
          const f2 Cy = f2_fma(Rz[u], dx, Rx[u] * ndz);
          const f2 Cz = f2_fma(Rx[u], dy, Ry[u] * ndx);
          const f2 e = f2_fma(Rz[u], Bz, f2_fma(Ry[u], By, Rx[u] * Bx));
          const f2 uu = ia[u] * ib;
          const f2 den = f2_fma(e, uu, one);
          const f2 w = uu * f2_rcp(den);
          const f2 s = (ia[u] + ib) * w;
          const f2 est = two - den;   // 1 - cos, error below 1e-6
          float r20, r21, s0, s1, e0, e1;
          f2_unpack(R2[u], r20, r21);
          f2_unpack(s, s0, s1);
          f2_unpack(est, e0, e1);
          bool far0 = r20 >= sg.far2.x && sg.id[0] >= 0, far1 = r21 >= sg.far2.y && sg.id[1] >= 0;
          bool ok0 = far0 && e0 > 2e-6f, ok1 = far1 && e1 > 2e-6f;
          bool sp0 = sg.id[0] >= 0 && !far0, sp1 = sg.id[1] >= 0 && !far1;
          if (__any_sync(0xffffffffu, (far0 && !ok0) || (far1 && !ok1))) {
            // near the colinearity cut-off: the exact 1 - cos = |C|^2 u w
            const f2 tc = f2_fma(Cz, Cz, f2_fma(Cy, Cy, Cx * Cx)) * (uu * w);
            float tc0, tc1;
            f2_unpack(tc, tc0, tc1);
            if (far0 && !ok0) {
              ok0 = tc0 > kColHi;
              sp0 = !ok0 && !(tc0 < kColLo);
            }
            if (far1 && !ok1) {
              ok1 = tc1 > kColHi;
              sp1 = !ok1 && !(tc1 < kColLo);
            }
          }
          const f2 sk = f2_pack(ok0 ? s0 : 0.f, ok1 ? s1 : 0.f);
          b[u][0] = f2_fma(Cx, sk, b[u][0]);
          b[u][1] = f2_fma(Cy, sk, b[u][1]);
          b[u][2] = f2_fma(Cz, sk, b[u][2]);
          if (sp0 || sp1) {
            if (sp0) special(u, sg.id[0]);
            if (sp1) special(u, sg.id[1]);
          }
          Rx[u] = Bx;
          Ry[u] = By;
          Rz[u] = Bz;
          R2[u] = B2;
          ia[u] = ib;
        }
      }
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
    // the segments that do not chain, two per record
    {
      f2 b[kTT][3];
#pragma unroll
      for (int u = 0; u < kTT; ++u) b[u][0] = b[u][1] = b[u][2] = f2_splat(0.f);
      for (int q = 0; 2 * q < n_irr; ++q) pair_interact<kTwo>(sh_irr[q], T, b, special);
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
  }
#pragma unroll
  for (int u = 0; u < kTT; ++u) {
    const int i = base + threadIdx.x + kPB * u;
    if (i >= n_t) continue;
    double* o = part + ((size_t)blockIdx.z * gridDim.y + j) * 3 * stride + 3 * (size_t)(order ? order[i] : i);
    const bool act = kk[u] >= 0;
    o[0] = act ? acc[u][0] : 0;
    o[1] = act ? acc[u][1] : 0;
    o[2] = act ? acc[u][2] : 0;
  }
}

// v_nl = part[0]; v_img = sum_j part[j] in image order (src/tangle.c:627-638);
// mirror images reflect their velocity (src/tangle.c:633-634).  With source
// splits, each image's partial sums are added split by split, in order.
__global__ void k_reduce_images(OvParams P, const double* __restrict__ part, int n_t,
                                double* v_nl, double* v_img, int splits) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_t) return;
  const size_t img_stride = 3 * (size_t)n_t, split_stride = img_stride * (P.n_img + 1);
  d3 a = ld3(part, k);
  for (int z = 1; z < splits; ++z) a = a + ld3(part + z * split_stride, k);
  if (v_nl) st3(v_nl, k, a);
  d3 s = mk3(0, 0, 0);
  for (int j = 1; j <= P.n_img; ++j) {
    d3 v = ld3(part + (size_t)j * img_stride, k);
    for (int z = 1; z < splits; ++z) v = v + ld3(part + z * split_stride + (size_t)j * img_stride, k);
    int face = P.img[j - 1][3];
    if (face > -1) v = mirror_dir(v, face);
    s = s + v;
  }
  if (v_img) st3(v_img, k, s);
}

__global__ void k_add3(const double* a, const double* b, double* o, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 3 * n) o[i] = a[i] + b[i];
}

}  // namespace

static bool ensure_segtab(ov_state_impl* s, const double* pos);
bool ov_segment_table(ov_state_impl* s, const double* pos) { return ensure_segtab(s, pos); }

static bool ensure_segtab(ov_state_impl* s, const double* pos) {
  if (!s->seg64.reserve(sizeof(double) * 6 * (size_t)s->n)) return false;
  if (!s->segid.reserve(sizeof(int) * (size_t)s->n)) return false;
  k_segtab<<<(s->n + 255) / 256, 256, 0, s->stream>>>(s->P, pos, s->links.as<int2>(),
                                                       s->status.as<int2>(), s->seg64.as<double>(),
                                                       s->segid.as<int>(), s->n);
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  return true;
}

// Source splits for a grid of `blocks` target blocks: enough that a small
// tangle still fills the GPU (about 4 blocks per SM), each split a whole
// number of tiles of `tile` sources; returns the sources per split.
static int source_chunk(int n_src, long long blocks, int tile, int* splits) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 1;
  }
  long long want = (4LL * sms + blocks - 1) / std::max(1LL, blocks);
  int sp = (int)std::min<long long>(16, std::max<long long>(1, want));
  int chunk = (n_src + sp - 1) / sp;
  chunk = std::max(tile, (chunk + tile - 1) / tile * tile);
  *splits = std::max(1, (n_src + chunk - 1) / chunk);
  return chunk;
}

bool ov_direct_nodes(ov_state_impl* s, const double* pos, double* v_nl, double* v_img) {
  if (s->n == 0) return true;
  if (!ensure_segtab(s, pos)) return false;
  int nimg = s->P.n_img;
  SegTab S{s->seg64.as<double>(), s->segid.as<int>()};
  OvStatsAcc& st = ov_stats_tls();
  int splits = 1;
  if (s->P.precision == OV_PREC_MIXED) {
    static const int chain_form = getenv("OV_DIRECT_CHAIN") ? atoi(getenv("OV_DIRECT_CHAIN")) : 0;
    // targets in key order from the tree's sort (timed as the build), or in
    // slot order for the two-float chain form, which needs no sort
    const bool slot_order = chain_form == 2;
    const int* order = nullptr;
    int n_t = s->n;
    if (!slot_order) {
      if (!ov_tree_build(s, pos, &s->tree)) return false;
      order = s->tree.perm.as<int>();
      n_t = s->tree.n_nodes;
    }
    if ((slot_order ? s->n_active : s->tree.n_nodes) == 0) {
      // every slot EMPTY: no targets and no segments
      cudaEventRecord(s->ev1, s->stream);
      cudaEventRecord(s->ev2, s->stream);
      OV_TRY_CUDA(cudaMemsetAsync(v_nl, 0, sizeof(double) * 3 * s->n, s->stream));
      OV_TRY_CUDA(cudaMemsetAsync(v_img, 0, sizeof(double) * 3 * s->n, s->stream));
      return true;
    }
    const int bx = (n_t + kPTgt - 1) / kPTgt;
    // sources: slots in slot order (chain forms) or the sorted active nodes
    const int n_src = chain_form ? s->n : s->tree.n_nodes;
    const int chunk = source_chunk(n_src, (long long)bx * (nimg + 1), kPSrc, &splits);
    if (!s->img_part.reserve(sizeof(double) * 3 * (size_t)s->n * (nimg + 1) * splits)) return false;
    cudaEventRecord(s->ev1, s->stream);
    if (chain_form == 2) {
      k_direct_mixed_chain<true><<<dim3(bx, nimg + 1, splits), kPB, 0, s->stream>>>(
          s->P, S, n_src, pos, s->status.as<int2>(), nullptr, n_t, s->n, s->img_part.as<double>(), chunk);
    } else if (chain_form) {
      k_direct_mixed_chain<false><<<dim3(bx, nimg + 1, splits), kPB, 0, s->stream>>>(
          s->P, S, n_src, pos, s->status.as<int2>(), order, n_t, s->n, s->img_part.as<double>(), chunk);
    } else {
      k_direct_mixed_pairs<<<dim3(bx, nimg + 1, splits), kPB, 0, s->stream>>>(
          s->P, S, n_src, pos, s->status.as<int2>(), order, n_t, s->n, s->img_part.as<double>(), chunk);
    }
    OV_LAUNCHED();
    OV_TRY_CUDA(cudaGetLastError());
    // k_direct_mixed_pairs wrote part[j][k] for slots k in the sorted set only;
    // EMPTY slots are never read by the epilogue, but zero them for hygiene
  } else {
    const int bx = (s->n + kTB - 1) / kTB;
    const int chunk = source_chunk(s->n, (long long)bx * (nimg + 1), kTS, &splits);
    if (!s->img_part.reserve(sizeof(double) * 3 * (size_t)s->n * (nimg + 1) * splits)) return false;
    cudaEventRecord(s->ev1, s->stream);
    k_direct64<<<dim3(bx, nimg + 1, splits), kTB, 0, s->stream>>>(
        s->P, S, s->n, nullptr, pos, s->status.as<int2>(), nullptr, s->n, s->img_part.as<double>(), chunk);
    OV_LAUNCHED();
    OV_TRY_CUDA(cudaGetLastError());
  }
  cudaEventRecord(s->ev2, s->stream);
  k_reduce_images<<<(s->n + 255) / 256, 256, 0, s->stream>>>(s->P, s->img_part.as<double>(), s->n,
                                                              v_nl, v_img, splits);
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  (void)st;
  return true;
}

bool ov_direct_points(ov_state_impl* s, const double* pos, int npts, const double* pts,
                      const int* skip, const int* only, int n_only, double* out_nl,
                      double* out_img) {
  if (npts <= 0) return true;
  if (!ensure_segtab(s, pos)) return false;
  int nimg = out_img ? s->P.n_img : 0;
  SegTab S{s->seg64.as<double>(), s->segid.as<int>()};
  int n_src = only ? n_only : s->n;
  // few points over many sources: split the sources so the GPU fills
  const int bx = (npts + kTB - 1) / kTB;
  int splits = 1;
  const int chunk = source_chunk(std::max(1, n_src), (long long)bx * (nimg + 1), kTS, &splits);
  size_t bytes = sizeof(double) * 3 * (size_t)npts * (nimg + 1) * splits;
  if (!s->img_part.reserve(bytes)) return false;
  dim3 grid(bx, nimg + 1, splits);
  k_direct64<<<grid, kTB, 0, s->stream>>>(s->P, S, n_src, only, pts, nullptr, skip, npts,
                                          s->img_part.as<double>(), chunk);
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  // out_nl = part[0]; out_img = image sum in table order (src/tangle.c:624-638),
  // each split's partial sums added in split order
  OvParams P = s->P;
  P.n_img = nimg;
  k_reduce_images<<<(npts + 255) / 256, 256, 0, s->stream>>>(P, s->img_part.as<double>(), npts,
                                                              out_nl, out_img, splits);
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  return true;
}

bool ov_add3(cudaStream_t st, const double* a, const double* b, double* out, int n) {
  if (n <= 0) return true;
  k_add3<<<(3 * n + 255) / 256, 256, 0, st>>>(a, b, out, n);
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  return true;
}

// The direct point query with caller-provided scratch (ov_noalloc.cu):
// segment table seg (6 doubles per node) and fwd (n ints), per-image partial
// sums part (3 doubles per point and image), image sums img (3 per point).
// Launches only, on `st`; out = the tangle's own sum + the image sum.
bool ov_direct_points_scratch(cudaStream_t st, const OvParams& P, const double* pos,
                              const int2* links, const int2* status, int n, int npts,
                              const double* pts, const int* skip, double* seg, int* fwd,
                              double* part, double* out, double* img) {
  if (n > 0) {
    k_segtab<<<(n + 255) / 256, 256, 0, st>>>(P, pos, links, status, seg, fwd, n);
    OV_LAUNCHED();
  }
  dim3 grid((npts + kTB - 1) / kTB, P.n_img + 1);
  k_direct64<<<grid, kTB, 0, st>>>(P, SegTab{seg, fwd}, n, nullptr, pts, nullptr, skip, npts, part,
                                   std::max(1, n));
  OV_LAUNCHED();
  k_reduce_images<<<(npts + 255) / 256, 256, 0, st>>>(P, part, npts, out, img, 1);
  OV_LAUNCHED();
  k_add3<<<(3 * npts + 255) / 256, 256, 0, st>>>(out, img, out, npts);
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  return true;
}
