// ov_pair.cuh - packed FP32 pairs for sm_100a: two single-precision values
// in one 64-bit register pair, operated on by Blackwell's f32x2 add, sub,
// mul and fma (one instruction for both halves).  The mixed-form direct
// Biot-Savart kernels evaluate two sources per instruction this way; the
// halves are split only for the transcendental approximations, compares and
// selects.
#pragma once

#include <cuda_runtime.h>

struct f2 {
  unsigned long long v;
};

__device__ __forceinline__ f2 f2_pack(float lo, float hi) {
  f2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ f2 f2_splat(float x) { return f2_pack(x, x); }
__device__ __forceinline__ void f2_unpack(f2 a, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(a.v));
}

__device__ __forceinline__ f2 operator+(f2 a, f2 b) {
  f2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ f2 operator-(f2 a, f2 b) {
  f2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
__device__ __forceinline__ f2 operator*(f2 a, f2 b) {
  f2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r.v) : "l"(a.v), "l"(b.v));
  return r;
}
// a * b + c, each half rounded once
__device__ __forceinline__ f2 f2_fma(f2 a, f2 b, f2 c) {
  f2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r.v) : "l"(a.v), "l"(b.v), "l"(c.v));
  return r;
}

// hardware approximations (relative error ~2^-22), flush-to-zero: the
// arguments here are squared lengths and 1 + cos, never denormal
__device__ __forceinline__ float rsqrt_approx(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ f2 f2_rsqrt(f2 a) {
  float lo, hi;
  f2_unpack(a, lo, hi);
  return f2_pack(rsqrt_approx(lo), rsqrt_approx(hi));
}
__device__ __forceinline__ f2 f2_rcp(f2 a) {
  float lo, hi;
  f2_unpack(a, lo, hi);
  return f2_pack(rcp_approx(lo), rcp_approx(hi));
}

// ----------------------------------------------------------------------
// Mixed-form direct sums, two sources per instruction.  Sources are staged
// two by two: each value of sources 2i and 2i+1 sits in one 64-bit pair,
// and each thread's kTT targets are broadcast into both halves of theirs.
// Per segment-target pair (R = r1 - r, d = r2 - r1, R' = R + d, a = |R|,
// b = |R'|):
//   u = 1/(ab), 1 + cos = 1 + (R.R') u, r = 1/(1 + cos), w = u r
//   v = kappa/4pi (1/a + 1/b) w (R x d)        (R x R' = R x d)
//   1 - cos = |R x d|^2 u w                    (no cancellation)
// which is the reference's segment formula (src/tangle.c:486-517) and its
// colinearity cut-off |cos - 1| < 1e-8, zero inside it.  Within 2.5e-3 of
// the cut-off (the FP32 rounding bound of |R x d|^2, see seg_vel32), or
// nearer than the source's far radius, the pair is left to the caller's
// FP64 path.

#ifndef OV_PAIR_TT
#define OV_PAIR_TT 2
#endif
constexpr int kTT = OV_PAIR_TT;   // targets per thread
constexpr float kColLo = 1e-8f * (1.0f - 2.5e-3f);
constexpr float kColHi = 1e-8f * (1.0f + 2.5e-3f);

// two staged sources (index 0 in the low halves, 1 in the high halves):
//   q0 = (ax ay) pairs   q1 = (az dx)   q2 = (dy dz)   q3 = (-dx -dy)
//   q4 = (-dz d2)   q5 = (far2, id) pairs
//   q6 = (lo parts of ax ay)   q7 = (lo part of az, |d|): two-float form
template <bool kTwo>
struct __align__(16) PairSrc {
  float4 q[kTwo ? 8 : 6];
};

// one source: offsets a = r1 - O (hi + lo), d = r2 - r1, FP32 far radius
struct SrcVals {
  float ax, ay, az, dx, dy, dz, far2;
  int id;
  float lx, ly, lz;
};

__device__ __forceinline__ SrcVals src_none() {
  // zero length far away: the formula gives exactly zero
  return SrcVals{1.0e4f, 1.0e4f, 1.0e4f, 0.f, 0.f, 0.f, 0.f, -1, 0.f, 0.f, 0.f};
}

// a source from FP64 offsets: hi = fl32(p), lo = fl32(p - hi)
__device__ __forceinline__ SrcVals src_from(double px, double py, double pz, double dx, double dy,
                                            double dz, double far2, int id) {
  const float hx = (float)px, hy = (float)py, hz = (float)pz;
  return SrcVals{hx, hy, hz, (float)dx, (float)dy, (float)dz, (float)far2, id,
                 (float)(px - hx), (float)(py - hy), (float)(pz - hz)};
}

template <bool kTwo>
__device__ __forceinline__ void stage_pair(PairSrc<kTwo>& o, const SrcVals& s0, const SrcVals& s1) {
  const float d20 = fmaf(s0.dx, s0.dx, fmaf(s0.dy, s0.dy, s0.dz * s0.dz));
  const float d21 = fmaf(s1.dx, s1.dx, fmaf(s1.dy, s1.dy, s1.dz * s1.dz));
  o.q[0] = make_float4(s0.ax, s1.ax, s0.ay, s1.ay);
  o.q[1] = make_float4(s0.az, s1.az, s0.dx, s1.dx);
  o.q[2] = make_float4(s0.dy, s1.dy, s0.dz, s1.dz);
  o.q[3] = make_float4(-s0.dx, -s1.dx, -s0.dy, -s1.dy);
  o.q[4] = make_float4(-s0.dz, -s1.dz, d20, d21);
  o.q[5] = make_float4(s0.far2, s1.far2, __int_as_float(s0.id), __int_as_float(s1.id));
  if constexpr (kTwo) {
    o.q[6] = make_float4(s0.lx, s1.lx, s0.ly, s1.ly);
    o.q[7] = make_float4(s0.lz, s1.lz, sqrtf(d20), sqrtf(d21));
  }
}

// Target offsets: hi and (two-float form) lo parts, broadcast into pairs.
struct PairTargets {
  f2 x[kTT], y[kTT], z[kTT];
  f2 lx[kTT], ly[kTT], lz[kTT];
};

__device__ __forceinline__ void set_target(PairTargets& t, int k, double px, double py, double pz) {
  const float hx = (float)px, hy = (float)py, hz = (float)pz;
  t.x[k] = f2_splat(hx);
  t.y[k] = f2_splat(hy);
  t.z[k] = f2_splat(hz);
  t.lx[k] = f2_splat((float)(px - hx));
  t.ly[k] = f2_splat((float)(py - hy));
  t.lz[k] = f2_splat((float)(pz - hz));
}

// Two sources against the thread's targets: FP32 contributions (without the
// kappa/4pi factor) into b[k] (low half: source 0, high half: source 1);
// pairs needing FP64 call special(k, id).  The two-float form takes R as
// (a_hi - t_hi) + (a_lo - t_lo), which carries ~2 ulps of |R| itself
// however far source and target are from the origin.  With kBound (two-
// float form only) eb[k] also accumulates |d| / |R|^2 over the pairs
// evaluated here in FP32, the quantity that bounds their rounding error.
template <bool kTwo, bool kBound, class Special>
__device__ __forceinline__ void pair_interact_impl(const PairSrc<kTwo>& src, const PairTargets& T,
                                                   f2 (&b)[kTT][3], Special&& special, f2 (&eb)[kTT]) {
  static_assert(kTwo || !kBound, "the error bound needs |d|, staged in the two-float form");
  const float4 q0 = src.q[0], q1 = src.q[1], q2 = src.q[2], q3 = src.q[3], q4 = src.q[4], q5 = src.q[5];
  const f2 ax = f2_pack(q0.x, q0.y), ay = f2_pack(q0.z, q0.w), az = f2_pack(q1.x, q1.y);
  const f2 dx = f2_pack(q1.z, q1.w), dy = f2_pack(q2.x, q2.y), dz = f2_pack(q2.z, q2.w);
  const f2 ndx = f2_pack(q3.x, q3.y), ndy = f2_pack(q3.z, q3.w), ndz = f2_pack(q4.x, q4.y);
  const f2 d2 = f2_pack(q4.z, q4.w);
  const f2 one = f2_splat(1.0f), two = f2_splat(2.0f);
  f2 alx, aly, alz, dn;
  if constexpr (kTwo) {
    const float4 q6 = src.q[6], q7 = src.q[7];
    alx = f2_pack(q6.x, q6.y);
    aly = f2_pack(q6.z, q6.w);
    alz = f2_pack(q7.x, q7.y);
    dn = f2_pack(q7.z, q7.w);
  }
#pragma unroll
  for (int k = 0; k < kTT; ++k) {
    f2 Rx = ax - T.x[k], Ry = ay - T.y[k], Rz = az - T.z[k];
    if constexpr (kTwo) {
      Rx = Rx + (alx - T.lx[k]);
      Ry = Ry + (aly - T.ly[k]);
      Rz = Rz + (alz - T.lz[k]);
    }
    const f2 R2 = f2_fma(Rz, Rz, f2_fma(Ry, Ry, Rx * Rx));
    const f2 Rd = f2_fma(Rz, dz, f2_fma(Ry, dy, Rx * dx));
    const f2 Q2 = f2_fma(two, Rd, R2 + d2);
    const f2 ia = f2_rsqrt(R2), ib = f2_rsqrt(Q2);
    const f2 u = ia * ib;
    const f2 r = f2_rcp(f2_fma(R2 + Rd, u, one));
    const f2 w = u * r;
    const f2 s = (ia + ib) * w;
    const f2 Cx = f2_fma(Ry, dz, Rz * ndy);
    const f2 Cy = f2_fma(Rz, dx, Rx * ndz);
    const f2 Cz = f2_fma(Rx, dy, Ry * ndx);
    const f2 tc = f2_fma(Cz, Cz, f2_fma(Cy, Cy, Cx * Cx)) * (u * w);   // 1 - cos
    float tc0, tc1, r20, r21, s0, s1;
    f2_unpack(tc, tc0, tc1);
    f2_unpack(R2, r20, r21);
    f2_unpack(s, s0, s1);
    const bool far0 = r20 >= q5.x, far1 = r21 >= q5.y;
    const bool ok0 = far0 && tc0 > kColHi, ok1 = far1 && tc1 > kColHi;
    // colinear (zero) and FP64 cases add nothing here
    const f2 sk = f2_pack(ok0 ? s0 : 0.f, ok1 ? s1 : 0.f);
    b[k][0] = f2_fma(Cx, sk, b[k][0]);
    b[k][1] = f2_fma(Cy, sk, b[k][1]);
    b[k][2] = f2_fma(Cz, sk, b[k][2]);
    if constexpr (kBound) {
      float i0, i1;
      f2_unpack(ia * ia, i0, i1);
      eb[k] = f2_fma(dn, f2_pack(ok0 ? i0 : 0.f, ok1 ? i1 : 0.f), eb[k]);
    }
    const bool sp0 = !ok0 && !(far0 && tc0 < kColLo);
    const bool sp1 = !ok1 && !(far1 && tc1 < kColLo);
    if (sp0 || sp1) {
      if (sp0) special(k, __float_as_int(q5.z));
      if (sp1) special(k, __float_as_int(q5.w));
    }
  }
}

template <bool kTwo, class Special>
__device__ __forceinline__ void pair_interact(const PairSrc<kTwo>& src, const PairTargets& T,
                                              f2 (&b)[kTT][3], Special&& special) {
  f2 unused[kTT];
  pair_interact_impl<kTwo, false>(src, T, b, special, unused);
}

// ----------------------------------------------------------------------
// Chain order: sources staged in slot order, where a loop's segments
// follow one another, so segment m runs from node m to node m + 1 for all
// but one segment per loop ("chained").  Each node's offset R = r_node - r,
// |R|^2 and 1/|R| are formed once per target and serve both segments that
// touch it.  Per pair (a = |R|, b = |R'|):
//   u = 1/(ab), den = 1 + R.R' u = 1 + cos, w = u / den
//   v = kappa/4pi (1/a + 1/b) w (R x d)
// R x d, with the segment vector d staged on its own, keeps the FP32 error
// of the cross product at a few ulps of |R||d|.  The reference's cut-off
// test (src/tangle.c:505-506) takes 1 - cos = |R x d|^2 u w, as in the
// two-source form.  That is 28 lane operations and 2 hardware
// approximations per interaction, against 31 and 3 for the two-source form
// above.  Segments that do not chain (a loop's closing segment, a segment
// wrapped across a periodic face) take the two-source form from a list.
//
// A tile holds kCH chained pairs: pair i is segments sb + i (low half) and
// sb + kCH + i (high half); node pack i is nodes sb + i and sb + kCH + i,
// i = 0 .. kCH.
constexpr int kCH = 64;

#ifndef OV_CHAIN_UNROLL
#define OV_CHAIN_UNROLL 4
#endif
constexpr int kChainUnroll = OV_CHAIN_UNROLL;

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


// node pack: two node offsets from the origin (hi, and lo parts in the
// two-float form); `valid` false places the node far away, used by no
// chained segment
template <bool kTwo>
__device__ __forceinline__ void chain_node_set(ChainNode<kTwo>& nd, const double (&off)[2][3],
                                               const bool (&valid)[2]) {
  float o[2][3], lo[2][3];
#pragma unroll
  for (int h = 0; h < 2; ++h)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      o[h][c] = valid[h] ? (float)off[h][c] : 1.0e4f;
      lo[h][c] = valid[h] ? (float)(off[h][c] - (double)o[h][c]) : 0.f;
    }
  nd.x = make_float2(o[0][0], o[1][0]);
  nd.y = make_float2(o[0][1], o[1][1]);
  nd.z = make_float2(o[0][2], o[1][2]);
  if constexpr (kTwo) {
    nd.lx[0] = make_float2(lo[0][0], lo[1][0]);
    nd.ly[0] = make_float2(lo[0][1], lo[1][1]);
    nd.lz[0] = make_float2(lo[0][2], lo[1][2]);
  }
}

// chained pair: segment vectors, FP32 far radii and slots (-1: none)
__device__ __forceinline__ void chain_seg_set(ChainSeg& sg, const float (&dd)[2][3], const float (&far2)[2],
                                              const int (&id)[2]) {
  sg.a = make_float4(dd[0][0], dd[1][0], dd[0][1], dd[1][1]);
  sg.b = make_float4(dd[0][2], dd[1][2], -dd[0][0], -dd[1][0]);
  sg.c = make_float4(-dd[0][1], -dd[1][1], -dd[0][2], -dd[1][2]);
  sg.far2 = make_float2(far2[0], far2[1]);
  sg.id[0] = id[0];
  sg.id[1] = id[1];
}

// The kCH chained pairs of a staged tile against the thread's targets:
// FP32 partial sums over 32 segments, each added (times f4pi) into acc;
// pairs needing FP64 call special(u, slot).  Every thread of the warp runs
// the same iterations.
template <bool kTwo, class Special>
__device__ __forceinline__ void chain_sweep(const ChainNode<kTwo>* sh_node, const ChainSeg* sh_seg,
                                            const PairTargets& T, double (&acc)[kTT][3], double f4pi,
                                            Special&& special) {
  const f2 one = f2_splat(1.0f);
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
        // 1 - cos = |C|^2 u w for every pair: far segments of a large
        // tangle subtend angles whose 1 - cos lies below any cheaper
        // estimate's error, so a pre-test on 2 - den decides almost none
        const f2 tc = f2_fma(Cz, Cz, f2_fma(Cy, Cy, Cx * Cx)) * (uu * w);
        float r20, r21, s0, s1, tc0, tc1;
        f2_unpack(R2[u], r20, r21);
        f2_unpack(s, s0, s1);
        f2_unpack(tc, tc0, tc1);
        const bool far0 = r20 >= sg.far2.x && sg.id[0] >= 0, far1 = r21 >= sg.far2.y && sg.id[1] >= 0;
        const bool ok0 = far0 && tc0 > kColHi, ok1 = far1 && tc1 > kColHi;
        // near pairs and pairs within the cut-off's rounding band: FP64
        const bool sp0 = sg.id[0] >= 0 && !ok0 && !(far0 && tc0 < kColLo);
        const bool sp1 = sg.id[1] >= 0 && !ok1 && !(far1 && tc1 < kColLo);
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
}
