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
                          mk3(sh_r[q][6], sh_r[q][7], sh_r[q][8]), r, P.col_cut);
      ax += v.x; ay += v.y; az += v.z;
    }
  }
  if (k < n_t) {
    double* o = part + ((size_t)blockIdx.z * gridDim.y + j) * 3 * n_t + 3 * (size_t)k;
    o[0] = act ? ax : 0; o[1] = act ? ay : 0; o[2] = act ? az : 0;
  }
}

// FP64 in chain order: sources in slot order, where a loop's segments
// follow one another (segment m runs from node m to its forward node m + 1
// for all but one segment per loop).  Each node's R = r_node - r, |R|^2 and
// refined 1/|R| are formed once per target and serve both segments that
// touch it, so a chained segment costs its R.R', one refined reciprocal and
// the cross product: about 42 FP64 operations against 55 for seg_vel64_nr.
// R' is r2 - r itself, as the reference forms it (src/tangle.c:490-491).
// The cut-offs are decided as in seg_vel64_nr: where |R| or |R'| is within
// 1.5e-8 or cos within 2e-8 of 1, the reference's own operations decide
// (seg_vel64).  Segments that do not chain (a loop's closing segment, one
// wrapped across a periodic face) take seg_vel64_nr from a list.  Block =
// kTB targets x one image; targets are node slots (status-filtered, skip =
// the slot) or explicit points (kPoints, skip from tskip).
constexpr int kCS = 128;   // chained segments per shared-memory tile
static_assert(kCS == kTS, "the chain sweep splits sources as k_direct64 does");

template <bool kPoints>
__global__ void __launch_bounds__(kTB) k_direct64_chain(OvParams P, SegTab S, int n_src,
                                                        const double* __restrict__ pos,
                                                        const double* __restrict__ tpos,
                                                        const int2* __restrict__ tstatus,
                                                        const int* __restrict__ tskip, int n_t,
                                                        double* __restrict__ part, int chunk) {
  __shared__ double sh_node[kCS + 1][3];
  __shared__ int sh_kind[kCS];   // 1: chained, 0: no segment or in the list
  __shared__ int sh_irr[kCS];
  __shared__ int sh_nirr;
  const int j = blockIdx.y;   // 0: the tangle itself, j >= 1: image j-1
  const int k = blockIdx.x * kTB + threadIdx.x;
  bool act = k < n_t;
  if (act && !kPoints) act = tstatus[k].x != OV_EMPTY && tstatus[k].x != OV_PINNED;
  d3 r = mk3(0, 0, 0);
  int skip = -1;
  if (act) {
    r = ld3(kPoints ? tpos : pos, k);
    if (j > 0) r = image_point(P, j - 1, r);
    else skip = kPoints ? (tskip ? tskip[k] : -1) : k;
  }
  double ax = 0, ay = 0, az = 0;
  const double f4pi = P.f4pi;
  const int s_lo = blockIdx.z * chunk, s_hi = min(n_src, s_lo + chunk);
  for (int sb = s_lo; sb < s_hi; sb += kCS) {
    __syncthreads();
    if (threadIdx.x == 0) sh_nirr = 0;
    __syncthreads();
    // nodes sb .. sb + kCS (positions; a slot beyond the range or EMPTY is
    // used by no chained segment)
    for (int i = threadIdx.x; i <= kCS; i += kTB) {
      const int m = sb + i;
      const d3 p = m < n_src ? ld3(pos, m) : mk3(0, 0, 0);
      sh_node[i][0] = p.x;
      sh_node[i][1] = p.y;
      sh_node[i][2] = p.z;
    }
    for (int i = threadIdx.x; i < kCS; i += kTB) {
      const int m = sb + i;
      const int fw = m < s_hi ? S.fwd[m] : -1;
      int kind = 0;
      if (fw >= 0) {
        const double* sg = S.r1r2 + 6 * (size_t)m;
        bool chained = fw == m + 1;
        if (chained) {
          const d3 e = ld3(pos, fw);
          chained = e.x == sg[3] && e.y == sg[4] && e.z == sg[5];
        }
        if (chained) kind = 1;
        else sh_irr[atomicAdd(&sh_nirr, 1)] = m;
      }
      sh_kind[i] = kind;
    }
    __syncthreads();
    if (!act) continue;
    // node 0 of the tile
    d3 Ra = mk3(sh_node[0][0], sh_node[0][1], sh_node[0][2]) - r;
    double Ra2 = dot3(Ra, Ra);
    double ia = Ra2 >= 2.25e-16 ? rsqrt_nr(Ra2) : 0.0;
    const int cnt = min(kCS, s_hi - sb);
#pragma unroll 2
    for (int i = 0; i < cnt; ++i) {
      const d3 nb = mk3(sh_node[i + 1][0], sh_node[i + 1][1], sh_node[i + 1][2]);
      const d3 Rb = nb - r;
      const double Rb2 = dot3(Rb, Rb);
      const double ib = Rb2 >= 2.25e-16 ? rsqrt_nr(Rb2) : 0.0;
      const int m = sb + i;
      // skip rule of calculate_vs_shift (src/tangle.c:567-569): segment m
      // runs from m to m + 1
      if (sh_kind[i] && m != skip && m + 1 != skip) {
        d3 v;
        const double RRp = dot3(Ra, Rb);
        const double u = ia * ib;
        if (Ra2 < 2.25e-16 || Rb2 < 2.25e-16 || fabs(fma(RRp, u, -1.0)) < 2.0 * P.col_cut) {
          v = seg_vel64(f4pi, mk3(sh_node[i][0], sh_node[i][1], sh_node[i][2]), nb, r, P.col_cut);
        } else {
          const double sc = f4pi * (ia + ib) * (u * rcp_nr(fma(RRp, u, 1.0)));
          v = cross3(Ra, Rb) * sc;
        }
        ax += v.x;
        ay += v.y;
        az += v.z;
      }
      Ra = Rb;
      Ra2 = Rb2;
      ia = ib;
    }
    // the segments that do not chain
    const int nirr = sh_nirr;
    for (int q = 0; q < nirr; ++q) {
      const int m = sh_irr[q];
      const int fw = S.fwd[m];
      if (m == skip || fw == skip) continue;
      const double* sg = S.r1r2 + 6 * (size_t)m;
      const d3 r1 = mk3(sg[0], sg[1], sg[2]), r2 = mk3(sg[3], sg[4], sg[5]);
      const d3 v = seg_vel64_nr(f4pi, r1, r2, r2 - r1, r, P.col_cut);
      ax += v.x;
      ay += v.y;
      az += v.z;
    }
  }
  if (k < n_t) {
    double* o = part + ((size_t)blockIdx.z * gridDim.y + j) * 3 * (size_t)n_t + 3 * (size_t)k;
    o[0] = act ? ax : 0;
    o[1] = act ? ay : 0;
    o[2] = act ? az : 0;
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
// interactions (targets x segments x (1 + images)) up to which the mixed
// direct sum runs in slot order without the key sort
#ifndef OV_SLOT_ORDER_WORK
#define OV_SLOT_ORDER_WORK 2e8
#endif
constexpr double kSlotOrderWork = OV_SLOT_ORDER_WORK;

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

// Mixed form in chain order for small sums (k_direct_mixed_chain, the sweep
// in ov_pair.cuh): sources in slot order, each tile's chained segments swept
// with shared end nodes and the others in the two-source form; targets in
// slot order with two-float offsets (hi + lo), so R carries ~2 ulps of |R|
// whatever a block's extent and no key sort is needed.  Measured: on a
// 4096-point ring an RK4 step takes less than the FP64 form's (the key sort
// of k_direct_mixed_pairs costs more than its sum there); on the 22.4k-point
// periodic tangle k_direct_mixed_pairs is faster (18.6 against 24.4 ms).
static_assert(2 * kCH == kPSrc, "a chain tile is the two-source form's tile");

#ifndef OV_DIRECT_CHAIN_MIN_BLOCKS
#define OV_DIRECT_CHAIN_MIN_BLOCKS 4
#endif
__global__ void __launch_bounds__(kPB, OV_DIRECT_CHAIN_MIN_BLOCKS) k_direct_mixed_chain(
    OvParams P, SegTab S, int n_src, const double* __restrict__ pos, const int2* __restrict__ tstatus,
    int n_t, double* __restrict__ part, int chunk) {
  __shared__ ChainNode<true> sh_node[kCH + 1];
  __shared__ ChainSeg sh_seg[kCH];
  __shared__ PairSrc<true> sh_irr[kPSrc / 2];
  __shared__ int sh_irr_id[kPSrc];
  __shared__ int sh_n_irr;
  const int j = blockIdx.y;   // 0: the tangle itself, j >= 1: image j-1
  const int base = blockIdx.x * kPTgt;
  // offsets from the coordinate origin (with two-float offsets the origin
  // costs no accuracy, and a slot may be EMPTY)
  const d3 O = mk3(0, 0, 0);
  int kk[kTT];
  PairTargets T;
#pragma unroll
  for (int u = 0; u < kTT; ++u) {
    const int i = base + threadIdx.x + kPB * u;
    int k = i < n_t ? i : -1;
    if (k >= 0 && (tstatus[k].x == OV_EMPTY || tstatus[k].x == OV_PINNED)) k = -1;
    kk[u] = k;
    d3 r = O;
    if (k >= 0) {
      r = ld3(pos, k);
      if (j > 0) r = image_point(P, j - 1, r);
    }
    set_target(T, u, r.x, r.y, r.z);
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
  for (int sb = s_lo; sb < s_hi; sb += kPSrc) {
    __syncthreads();
    if (threadIdx.x == 0) sh_n_irr = 0;
    __syncthreads();
    // node packs: nodes sb + i and sb + kCH + i (EMPTY or beyond the range:
    // far away, used by no chained segment)
    for (int i = threadIdx.x; i <= kCH; i += kPB) {
      double off[2][3];
      bool valid[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int m = sb + i + h * kCH;
        valid[h] = m < n_src && tstatus[m].x != OV_EMPTY;
        const d3 p = valid[h] ? ld3(pos, m) : O;
        off[h][0] = p.x - O.x;
        off[h][1] = p.y - O.y;
        off[h][2] = p.z - O.z;
      }
      chain_node_set<true>(sh_node[i], off, valid);
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
      chain_seg_set(sh_seg[i], dd, f2v, idv);
    }
    __syncthreads();
    const int n_irr = sh_n_irr;
    for (int q = threadIdx.x; 2 * q < n_irr; q += kPB)
      stage_pair(sh_irr[q], stage_slot(sh_irr_id[2 * q]), 2 * q + 1 < n_irr ? stage_slot(sh_irr_id[2 * q + 1])
                                                                             : src_none());
    __syncthreads();
    chain_sweep<true>(sh_node, sh_seg, T, acc, f4pi, special);
    // the segments that do not chain, two per record
    {
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
  }
#pragma unroll
  for (int u = 0; u < kTT; ++u) {
    const int i = base + threadIdx.x + kPB * u;
    if (i >= n_t) continue;
    double* o = part + ((size_t)blockIdx.z * gridDim.y + j) * 3 * (size_t)n_t + 3 * (size_t)i;
    const bool act = kk[u] >= 0;
    o[0] = act ? acc[u][0] : 0;
    o[1] = act ? acc[u][1] : 0;
    o[2] = act ? acc[u][2] : 0;
  }
}

// Mixed form at explicit points, with a bound on its rounding error.  The
// reconnection pass (src/vortex_dynamics.c:266-281) needs only the sign of
// its approach test from these sums, so each point also gets
//   E = kMixedBoundU * kappa/4pi * sum |d| / |R|^2
// over the pairs evaluated in FP32 (all others take the FP64 formula, and
// the colinear ones are zero in both), which bounds |mixed - FP64| of the
// tangle's own sum plus its image sum.  Per FP32 pair, with u = 2^-24, a
// far pair (|R| >= 4 |d|) and |v| <= 1.6 kappa/4pi |d| / |R|^2:
//   - inputs: the two-float R carries <= 4u |R|, d <= 2u |d|; the formula's
//     sensitivity turns these into <= 28u kappa/4pi |d| / |R|^2;
//   - evaluation: ~20 FP32 roundings plus rsqrt.approx (2^-22.9) and
//     rcp.approx (1 ulp), the cross product's absolute error <= 2u |R||d|
//     per component: <= 25u kappa/4pi |d| / |R|^2;
//   - the FP32 partial sums of 16 terms per half: <= 26u of the sum of
//     |v| over those terms.
// Together <= 79u; kMixedBoundU = 256u leaves a factor of three.
// Targets: explicit points, two-float offsets from the coordinate origin
// (so a batch of points anywhere in the box keeps R to a few ulps of |R|),
// skip[i] the slot whose own segments the tangle's sum leaves out.
constexpr double kMixedBoundU = 256.0 / 16777216.0;

__global__ void __launch_bounds__(kPB) k_direct_mixed_points(OvParams P, SegTab S, int n_src,
                                                             const double* __restrict__ pos,
                                                             const double* __restrict__ tpos,
                                                             const int* __restrict__ tskip, int n_t,
                                                             double* __restrict__ part,
                                                             double* __restrict__ bpart, int chunk) {
  __shared__ PairSrc<true> sh[kPSrc / 2];
  const int j = blockIdx.y;   // 0: the tangle itself, j >= 1: image j-1
  const int base = blockIdx.x * kPTgt;
  bool act[kTT];
  int kk[kTT];
  d3 rr[kTT];
  PairTargets T;
#pragma unroll
  for (int u = 0; u < kTT; ++u) {
    const int i = base + threadIdx.x + kPB * u;
    act[u] = i < n_t;
    d3 r = act[u] ? ld3(tpos, i) : mk3(0, 0, 0);
    if (act[u] && j > 0) r = image_point(P, j - 1, r);
    rr[u] = r;
    kk[u] = act[u] && j == 0 && tskip ? tskip[i] : -1;
    set_target(T, u, r.x, r.y, r.z);
  }
  double acc[kTT][3], eacc[kTT];
#pragma unroll
  for (int u = 0; u < kTT; ++u) acc[u][0] = acc[u][1] = acc[u][2] = eacc[u] = 0;
  const double f4pi = P.f4pi;
  // FP64 evaluation of segment id at target u, with the skip rule of
  // calculate_vs_shift (src/tangle.c:567-569) for the tangle itself
  auto special = [&](int u, int id) {
#pragma unroll
    for (int v = 0; v < kTT; ++v) {
      if (v != u) continue;
      if (!act[v] || id < 0) return;
      const int fw = S.fwd[id];
      if (j == 0 && (id == kk[v] || fw == kk[v])) return;
      const double* sg = S.r1r2 + 6 * (size_t)id;
      const d3 vv = seg_vel64(f4pi, mk3(sg[0], sg[1], sg[2]), mk3(sg[3], sg[4], sg[5]), rr[v]);
      acc[v][0] += vv.x;
      acc[v][1] += vv.y;
      acc[v][2] += vv.z;
    }
  };
  const int s_lo = blockIdx.z * chunk, s_hi = min(n_src, s_lo + chunk);
  // sources in slot order; the tangle's own segments wrapped across a
  // periodic face go to FP64, where the skip rule applies
  auto stage_one = [&](int m) -> SrcVals {
    const int fw = m < s_hi ? S.fwd[m] : -1;
    if (fw < 0) return src_none();
    const double* sg = S.r1r2 + 6 * (size_t)m;
    const double dxx = sg[3] - sg[0], dyy = sg[4] - sg[1], dzz = sg[5] - sg[2];
    double far2 = fmax(16.0 * (dxx * dxx + dyy * dyy + dzz * dzz), P.near2);
    if (j == 0) {
      const d3 e = ld3(pos, fw);
      if (e.x != sg[3] || e.y != sg[4] || e.z != sg[5]) far2 = 1e30;
    }
    return src_from(sg[0], sg[1], sg[2], dxx, dyy, dzz, far2, m);
  };
  for (int sb = s_lo; sb < s_hi; sb += kPSrc) {
    __syncthreads();
    for (int q = threadIdx.x; q < kPSrc / 2; q += kPB)
      stage_pair(sh[q], stage_one(sb + 2 * q), stage_one(sb + 2 * q + 1));
    __syncthreads();
    for (int q0 = 0; q0 < kPSrc / 2; q0 += 16) {
      f2 b[kTT][3], eb[kTT];
#pragma unroll
      for (int k = 0; k < kTT; ++k) b[k][0] = b[k][1] = b[k][2] = eb[k] = f2_splat(0.f);
#pragma unroll 2
      for (int q = q0; q < q0 + 16; ++q) pair_interact_impl<true, true>(sh[q], T, b, special, eb);
#pragma unroll
      for (int k = 0; k < kTT; ++k) {
        float lo, hi;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          f2_unpack(b[k][c], lo, hi);
          acc[k][c] += f4pi * ((double)lo + (double)hi);
        }
        f2_unpack(eb[k], lo, hi);
        eacc[k] += (double)lo + (double)hi;
      }
    }
  }
#pragma unroll
  for (int u = 0; u < kTT; ++u) {
    const int i = base + threadIdx.x + kPB * u;
    if (i >= n_t) continue;
    const size_t slab = (size_t)blockIdx.z * gridDim.y + j;
    double* o = part + slab * 3 * (size_t)n_t + 3 * (size_t)i;
    o[0] = acc[u][0];
    o[1] = acc[u][1];
    o[2] = acc[u][2];
    bpart[slab * (size_t)n_t + i] = eacc[u];
  }
}

// bound[i] = kMixedBoundU * kappa/4pi * (sum over splits and images of bpart)
__global__ void k_reduce_bounds(double f4pi, const double* __restrict__ bpart, int n_t, int slabs,
                                double* bound) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_t) return;
  double e = 0;
  for (int z = 0; z < slabs; ++z) e += bpart[(size_t)z * n_t + i];
  bound[i] = kMixedBoundU * f4pi * e;
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

// resident blocks per SM of a kernel at a block size (0 when unknown)
template <class K>
static int resident_blocks(K kernel, int threads) {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, threads, 0) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return nb;
}

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
// tangle still fills the GPU (about `per_sm` blocks per SM, at most
// `max_splits` splits), each split a whole number of tiles of `tile`
// sources; returns the sources per split.
//
// With `resident` (the kernel's resident blocks per SM) the split count is
// then raised, by at most 4x, to the one whose last wave of blocks is
// fullest: the blocks of one launch all take the same time, so a grid of
// 3.2 waves runs as long as 4.  (On the 22.4k-point tangle the two-source
// form had 2376 blocks against 740 resident, 20% of its time in the last,
// partly empty wave.)
static int source_chunk(int n_src, long long blocks, int tile, int* splits, int per_sm = 4,
                        int max_splits = 16, int resident = 0) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 1;
  }
  long long want = ((long long)per_sm * sms + blocks - 1) / std::max(1LL, blocks);
  int sp = (int)std::min<long long>(max_splits, std::max<long long>(1, want));
  if (resident > 0) {
    const int tiles = std::max(1, (n_src + tile - 1) / tile);   // at least a tile per split
    const int top = std::min(std::min(max_splits, 4 * sp), std::max(sp, tiles));
    const double slots = (double)resident * sms;
    double best = -1;
    int best_sp = sp;
    for (int c = sp; c <= top; ++c) {
      const double waves = (double)blocks * c / slots;
      const double fill = waves / std::ceil(waves);
      if (fill > best + 1e-3) {
        best = fill;
        best_sp = c;
      }
    }
    sp = best_sp;
  }
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
    // small sums: slot order, no key sort (k_direct_mixed_chain); otherwise
    // key order from the tree's sort (timed as the build)
    const double work = (double)s->n_targets * (double)s->n_segments * (1 + nimg);
    const bool slot_order = work <= kSlotOrderWork;
    int n_t = s->n;
    if (!slot_order) {
      if (!ov_tree_build(s, pos, &s->tree)) return false;
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
    // sources: every slot in slot order, or the sorted active nodes
    const int n_src = slot_order ? s->n : s->tree.n_nodes;
    static const int res_chain = resident_blocks(k_direct_mixed_chain, kPB);
    static const int res_pairs = resident_blocks(k_direct_mixed_pairs, kPB);
    const int chunk = source_chunk(n_src, (long long)bx * (nimg + 1), kPSrc, &splits, 4, 16,
                                   slot_order ? res_chain : res_pairs);
    if (!s->img_part.reserve(sizeof(double) * 3 * (size_t)s->n * (nimg + 1) * splits)) return false;
    cudaEventRecord(s->ev1, s->stream);
    if (slot_order) {
      k_direct_mixed_chain<<<dim3(bx, nimg + 1, splits), kPB, 0, s->stream>>>(
          s->P, S, n_src, pos, s->status.as<int2>(), n_t, s->img_part.as<double>(), chunk);
    } else {
      k_direct_mixed_pairs<<<dim3(bx, nimg + 1, splits), kPB, 0, s->stream>>>(
          s->P, S, n_src, pos, s->status.as<int2>(), s->tree.perm.as<int>(), n_t, s->n,
          s->img_part.as<double>(), chunk);
    }
    OV_LAUNCHED();
    OV_TRY_CUDA(cudaGetLastError());
    // k_direct_mixed_pairs wrote part[j][k] for slots k in the sorted set only;
    // EMPTY slots are never read by the epilogue, but zero them for hygiene
  } else {
    const int bx = (s->n + kTB - 1) / kTB;
    static const int res64 = resident_blocks(k_direct64_chain<false>, kTB);
    const int chunk = source_chunk(s->n, (long long)bx * (nimg + 1), kCS, &splits, 4, 16, res64);
    if (!s->img_part.reserve(sizeof(double) * 3 * (size_t)s->n * (nimg + 1) * splits)) return false;
    cudaEventRecord(s->ev1, s->stream);
    k_direct64_chain<false><<<dim3(bx, nimg + 1, splits), kTB, 0, s->stream>>>(
        s->P, S, s->n, pos, nullptr, s->status.as<int2>(), nullptr, s->n, s->img_part.as<double>(), chunk);
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
  // few points over many sources: split the sources so the GPU fills, about
  // four waves of the kernel's 7 resident blocks per SM
  const int bx = (npts + kTB - 1) / kTB;
  int splits = 1;
  static const int res64 = resident_blocks(k_direct64_chain<true>, kTB);
  const int chunk = source_chunk(std::max(1, n_src), (long long)bx * (nimg + 1), kTS, &splits, 32, 64, res64);
  size_t bytes = sizeof(double) * 3 * (size_t)npts * (nimg + 1) * splits;
  if (!s->img_part.reserve(bytes)) return false;
  dim3 grid(bx, nimg + 1, splits);
  if (only) {
    k_direct64<<<grid, kTB, 0, s->stream>>>(s->P, S, n_src, only, pts, nullptr, skip, npts,
                                            s->img_part.as<double>(), chunk);
  } else {
    // all segments: the chain sweep over slot order (kCS == kTS: same splits)
    k_direct64_chain<true><<<grid, kTB, 0, s->stream>>>(s->P, S, n_src, pos, pts, nullptr, skip, npts,
                                                        s->img_part.as<double>(), chunk);
  }
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

bool ov_direct_points_bounded(ov_state_impl* s, const double* pos, int npts, const double* pts,
                              const int* skip, double* out_nl, double* out_img, double* out_bound) {
  if (npts <= 0) return true;
  if (!ensure_segtab(s, pos)) return false;
  const int nimg = s->P.n_img;
  SegTab S{s->seg64.as<double>(), s->segid.as<int>()};
  const int bx = (npts + kPTgt - 1) / kPTgt;
  int splits = 1;
  // a few thousand points: about eight waves of the kernel's 4 resident
  // blocks per SM, so the last wave's tail is a small share
  static const int res_pts = resident_blocks(k_direct_mixed_points, kPB);
  const int chunk = source_chunk(std::max(1, s->n), (long long)bx * (nimg + 1), kPSrc, &splits, 32, 64, res_pts);
  const size_t slabs = (size_t)(nimg + 1) * splits;
  // per-image partial sums (3 per point) followed by the bound partials
  if (!s->img_part.reserve(sizeof(double) * 4 * (size_t)npts * slabs)) return false;
  double* part = s->img_part.as<double>();
  double* bpart = part + 3 * (size_t)npts * slabs;
  k_direct_mixed_points<<<dim3(bx, nimg + 1, splits), kPB, 0, s->stream>>>(s->P, S, s->n, pos, pts, skip, npts,
                                                                          part, bpart, chunk);
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  k_reduce_images<<<(npts + 255) / 256, 256, 0, s->stream>>>(s->P, part, npts, out_nl, out_img, splits);
  OV_LAUNCHED();
  k_reduce_bounds<<<(npts + 255) / 256, 256, 0, s->stream>>>(s->P.f4pi, bpart, npts, (int)slabs, out_bound);
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
