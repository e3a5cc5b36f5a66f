// ov_walk.cu - Barnes-Hut velocity walk (octree_get_vs, src/octree.c:275-343)
// for every node and every boundary image (src/tangle.c:605-609,627-636).
//
// Warp-coherent, stackless traversal: the cells are in depth-first preorder,
// so each lane only keeps the index of the next cell it must visit (c + 1
// after opening c, c.skip otherwise).  The warp visits the smallest of its
// lanes' next cells; lanes whose next cell it is take their own decision, so
// every lane evaluates exactly the interactions the reference's recursion
// would, and the warp's 32 targets (consecutive in key order, hence close in
// space) share every cell load.
//
// Decision per cell (reference order): N == 1 or min side < BH_grain ->
// direct sum over the cell's nodes; |r - com|/(wrapped) passes the opening
// test -> monopole + the reference's second-order terms; otherwise descend.
// The opening test compares the squared distance, computed with the
// reference's exact operations, against a per-cell threshold equivalent to
// Lm / d < theta in FP64.
//
// FP64 form: everything in FP64.  Mixed form: the expansion and far direct
// segments in FP32 from FP64-formed relative vectors, FP64 sums; the opening
// test and near segments (|R| < 4 |ds|) in FP64.
#include <float.h>

#include <algorithm>
#include <cmath>

#include "ov_internal.h"
#include "ov_pair.cuh"

namespace {

struct TreeView {
  const Cell* cells;
  const double* cell_lm;   // max box side per cell (opening test at a user theta)
  const int2* cell_range;  // first sorted node and count per cell
  const double* nodes64;   // per sorted node: r1, wrapped r2
  const int2* nodeids;     // per sorted node: slot, forward slot
  int n_cells;
  int n_nodes;
};

// squared distance from r to the cell's centre of mass after the reference's
// one-box wrap of the centre (seg_pwrap + segment_len, src/octree.c:286-287),
// with exactly its FP64 operations
__device__ __forceinline__ double mac_dist2(const OvParams& P, d3 r, double cx, double cy, double cz) {
  double u[3];
  const double rr[3] = {r.x, r.y, r.z};
  const double cc[3] = {cx, cy, cz};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double c = cc[a];
    if (P.periodic[a]) {
      double d = __dsub_rn(c, rr[a]);
      if (d > P.L[a] * 0.5) c = __dsub_rn(c, P.L[a]);
      else if (d < -P.L[a] * 0.5) c = __dadd_rn(c, P.L[a]);
    }
    u[a] = __dsub_rn(rr[a], c);
  }
  double s = __dmul_rn(u[0], u[0]);
  s = __dadd_rn(s, __dmul_rn(u[1], u[1]));
  s = __dadd_rn(s, __dmul_rn(u[2], u[2]));
  return s;
}

// The reference's expansion (src/octree.c:303-328), moments pre-scaled by
// kappa/4pi: gam x R / |R|^3 + (M21, 0, 0) / |R|^3 + (M.2 R_z) x R / |R|^5,
// where (M.2 R_z) = (M02 Rz, M12 Rz, M22 Rz) is what its mat3_vmul returns.
// Since (M.2 R_z) x R / |R|^5 = ((M.2) R_z / |R|^2) x R / |R|^3, the sum is
// ((gam + M.2 R_z / |R|^2) x R + (M21, 0, 0)) / |R|^3: one cross product.
// m = (M21, M02, M12, M22).
__device__ __forceinline__ d3 expansion64(const double* g, const double* m, d3 R) {
  const double R2 = dot3(R, R);
  const double inv = rsqrt(R2);
  const double inv2 = inv * inv;
  const double i3 = inv2 * inv;
  const double w = R.z * inv2;
  const d3 G = mk3(fma(m[1], w, g[0]), fma(m[2], w, g[1]), fma(m[3], w, g[2]));
  const d3 c = cross3(G, R);
  return mk3((c.x + m[0]) * i3, c.y * i3, c.z * i3);
}

__device__ __forceinline__ void expansion32(float g0, float g1, float g2, float m21, float m02,
                                            float m12, float m22, float Rx, float Ry, float Rz,
                                            float& vx, float& vy, float& vz) {
  const float R2 = fmaf(Rx, Rx, fmaf(Ry, Ry, Rz * Rz));
  const float inv = rsqrtf(R2);
  const float inv2 = inv * inv;
  const float i3 = inv2 * inv;
  const float w = Rz * inv2;
  const float Gx = fmaf(m02, w, g0), Gy = fmaf(m12, w, g1), Gz = fmaf(m22, w, g2);
  vx = fmaf(Gy, Rz, fmaf(-Gz, Ry, m21)) * i3;
  vy = fmaf(Gz, Rx, -Gx * Rz) * i3;
  vz = fmaf(Gx, Ry, -Gy * Rx) * i3;
}

__device__ __forceinline__ void prefetch_l1(const void* p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

enum { ACT_NONE = 0, ACT_P2P1 = 1, ACT_P2PN = 2, ACT_FAR = 3, ACT_OPEN = 4 };

// One segment at rp: FP64 with the reference's cut-offs, or (mixed, far
// segments |R| >= 4 |ds|) FP32 from FP64-formed R and ds.
template <bool kMixed>
__device__ __forceinline__ void p2p_one(const OvParams& P, d3 r1, d3 r2, d3 rp, double& ax,
                                        double& ay, double& az) {
  if (kMixed) {
    d3 R = r1 - rp;
    d3 ds = r2 - r1;
    double R2 = dot3(R, R), ds2 = dot3(ds, ds);
    float vx, vy, vz;
    if (R2 >= 16.0 * ds2 && ds2 > 0 &&
        seg_vel32((float)P.f4pi, (float)R.x, (float)R.y, (float)R.z, (float)ds.x, (float)ds.y,
                  (float)ds.z, vx, vy, vz)) {
      ax += vx; ay += vy; az += vz;
      return;
    }
  }
  d3 v = seg_vel64(P.f4pi, r1, r2, rp);
  ax += v.x; ay += v.y; az += v.z;
}

// One walk of one warp: lane target rp (valid if `live`), skip rule `skip`.
// Each visited cell is one 128-byte record, loaded once for the warp; both
// possible successors (first child q+1 and skip) are prefetched into L1.
template <bool kMixed>
__device__ d3 warp_walk(const OvParams& P, const TreeView& T, d3 rp, bool live, int skip,
                        bool use_thr, double theta, unsigned long long& n_p2p,
                        unsigned long long& n_far, unsigned long long& n_iter) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  int next = live ? 0 : T.n_cells;
  double ax = 0, ay = 0, az = 0;
  for (;;) {
    const int q = (int)__reduce_min_sync(FULL, (unsigned)next);
    if (q >= T.n_cells) break;
    const Cell* cp = T.cells + q;
    if (lane == 0 && q + 1 < T.n_cells) prefetch_l1(cp + 1);
    const int4 h = *reinterpret_cast<const int4*>(cp);              // a, b, skip, meta
    const double2 t0 = *reinterpret_cast<const double2*>(&cp->thr);  // thr, x0
    const double2 t1 = *reinterpret_cast<const double2*>(&cp->x[1]); // x1, x2
    const int kind = cell_kind(h.w);
    const int skp = h.z;
    if (lane == 1 && skp < T.n_cells) prefetch_l1(T.cells + skp);
    int act = ACT_NONE;
    if (next == q) {
      if (kind == CELL_LEAF1) {
        act = ACT_P2P1;
      } else if (kind == CELL_LEAFN) {
        act = ACT_P2PN;
      } else {
        double s = mac_dist2(P, rp, t0.y, t1.x, t1.y);
        bool pass = use_thr ? (s >= t0.x)
                            : (s > 0 && __ddiv_rn(T.cell_lm[q], __dsqrt_rn(s)) < theta);
        if (pass) act = ACT_FAR;
        else if (kind == CELL_OPEN) act = ACT_OPEN;
        else if (kind == CELL_OPEN_P2P) act = ACT_P2PN;
      }
      // every lane's next cell strictly increases, so a walk ends within
      // n_cells iterations whatever the cell records hold
      next = (act == ACT_OPEN) ? q + 1 : max(skp, q + 1);
    }
    if (act == ACT_FAR) {
      if (kMixed) {
        // bytes 104-127 are 8-byte aligned: three float2 loads
        const float2 f0 = *reinterpret_cast<const float2*>(&cp->f_g[0]);  // g0 g1
        const float2 f1 = *reinterpret_cast<const float2*>(&cp->f_g[2]);  // g2 m02
        const float2 f2 = *reinterpret_cast<const float2*>(&cp->f_m12);   // m12 m22
        float vx, vy, vz;
        expansion32(f0.x, f0.y, f1.x, __int_as_float(h.x), f1.y, f2.x, f2.y, (float)(rp.x - t0.y),
                    (float)(rp.y - t1.x), (float)(rp.z - t1.y), vx, vy, vz);
        ax += vx; ay += vy; az += vz;
      } else {
        d3 v = expansion64(cp->y, cp->m, mk3(rp.x - t0.y, rp.y - t1.x, rp.z - t1.y));
        ax += v.x; ay += v.y; az += v.z;
      }
    } else if (act == ACT_P2P1) {
      // skip rule of calculate_vs_shift (src/tangle.c:567-569)
      if (h.y != -1 && h.x != skip && h.y != skip)
        p2p_one<kMixed>(P, mk3(t0.y, t1.x, t1.y), mk3(cp->y[0], cp->y[1], cp->y[2]), rp, ax, ay, az);
    }
    const unsigned far_mask = __ballot_sync(FULL, act == ACT_FAR);
    const unsigned p1_mask = __ballot_sync(FULL, act == ACT_P2P1);
    const unsigned pn_mask = __ballot_sync(FULL, act == ACT_P2PN);
    if (lane == 0) {
      n_far += __popc(far_mask);
      n_p2p += __popc(p1_mask);
      ++n_iter;
    }
    if (pn_mask) {
      const int2 rg = T.cell_range[q];
      const int end = min(rg.x + rg.y, T.n_nodes);
      if (lane == 0) n_p2p += (unsigned long long)__popc(pn_mask) * rg.y;
      for (int i = max(rg.x, 0); i < end; ++i) {
        const int2 id = T.nodeids[i];
        if (act != ACT_P2PN) continue;
        if (id.y == -1 || id.x == skip || id.y == skip) continue;
        const double* nd = T.nodes64 + 6 * (size_t)i;
        p2p_one<kMixed>(P, mk3(nd[0], nd[1], nd[2]), mk3(nd[3], nd[4], nd[5]), rp, ax, ay, az);
      }
    }
  }
  return mk3(ax, ay, az);
}

// ----------------------------------------------------------------------
// Multi-image walk (tables of periodic shifts in {-1,0,1}^3, no mirrors).
//
// The reference walks the tree once per image point r - L s (27 walks for
// periodic-26), each with its own opening decisions, because the opening
// distance is |r - L s - com| after a single box wrap of the centre of mass
// (src/octree.c:286).  Per axis that distance is the minimum image for s = 0
// and either the same value or a larger one for s = +-1, so every image's
// walk visits a subset of the cells of the s = 0 walk.  One traversal per
// target therefore serves all images: each lane keeps, per tree level, the
// 27-bit mask of images that opened the parent, makes each image's decision
// exactly as the reference would (per-axis wrapped distances with its FP64
// operations), evaluates every image that accepts the cell or reaches a leaf
// from the same cell load, and descends while any image opens.
//
// combo c = 9 (sx+1) + 3 (sy+1) + (sz+1); c = 13 is the tangle itself.

constexpr int kCombos = 27;
constexpr int kPrimary = 13;
// up to this many open images besides the target's own are decided one by
// one; more take all 27 decisions at once (mac_exact)
constexpr int kFewImages = 4;
constexpr unsigned kAllImages = (1u << 27) - 1;
constexpr int kLevelSlots = 34;
constexpr int kMultiWarps = 4;

// Parameters of the walk's shortcut decisions (every image from the
// target's own distance): on = no image shifts along a non-periodic axis
// (whose images may lie nearer than the target); hw[a] = the largest
// |c - r| along axis a at which every image's wrap still undoes its shift
// (half a box less a rounding allowance; DBL_MAX on axes without shifts).
struct ImageShortcut {
  double hw[3];
  double half[3];   // L / 2 on periodic axes (the reference's wrap test), DBL_MAX otherwise
  int on;
};

// wrapped component u and its square for one image coordinate v
__device__ __forceinline__ double wrapped_sq(const OvParams& P, int a, double v, double c) {
  double cc = c;
  if (P.periodic[a]) {
    double d = __dsub_rn(c, v);
    if (d > P.L[a] * 0.5) cc = __dsub_rn(c, P.L[a]);
    else if (d < -P.L[a] * 0.5) cc = __dadd_rn(c, P.L[a]);
  }
  double u = __dsub_rn(v, cc);
  return __dmul_rn(u, u);
}

__device__ __forceinline__ float sel3f(int i, float a, float b, float c) {
  return i == 0 ? a : (i == 1 ? b : c);
}

// FP64 reference formula for one segment at one image point, and the FP64
// expansion at one image offset.  Inlined: out of line (__noinline__) the
// calls' register saves made the mixed walk 52.1 ms per launch at 1M points
// against 37.9 ms.
__device__ __forceinline__ d3 seg64_at(double f4pi, d3 r1, d3 r2, d3 t) { return seg_vel64(f4pi, r1, r2, t); }
__device__ __forceinline__ d3 expansion64_at(const Cell* cp, d3 R) { return expansion64(cp->y, cp->m, R); }

// One segment r1 -> r2 for every image in `mask`: FP64 with the reference's
// cut-offs and skip rule (the skip applies to the tangle itself only), or in
// the mixed form FP32 beyond the near radius.  Images are visited as nine
// (x, y) columns of three z shifts, the z loop unrolled.
// image coordinate r - L s along one axis, s = i - 1, with the reference's
// single rounding (shifted, src/tangle.c:51-53)
__device__ __forceinline__ double img_coord(double r, double L, int i) {
  return i == 1 ? r : (i == 0 ? __dsub_rn(r, -L) : __dsub_rn(r, L));
}

// The 27 opening decisions of a cell (wrapped squared distance of each
// image point to the centre of mass >= thr), exactly with the reference's
// FP64 operations: per axis and shift the wrapped square, summed x + y then
// + z as segment_len does (src/octree.c:284-296).  All 27 are independent.
__device__ __forceinline__ unsigned mac_exact(const OvParams& P, d3 r, double cx, double cy,
                                              double cz, double thr) {
  const double qx[3] = {wrapped_sq(P, 0, img_coord(r.x, P.L[0], 0), cx), wrapped_sq(P, 0, r.x, cx),
                        wrapped_sq(P, 0, img_coord(r.x, P.L[0], 2), cx)};
  const double qy[3] = {wrapped_sq(P, 1, img_coord(r.y, P.L[1], 0), cy), wrapped_sq(P, 1, r.y, cy),
                        wrapped_sq(P, 1, img_coord(r.y, P.L[1], 2), cy)};
  const double qz[3] = {wrapped_sq(P, 2, img_coord(r.z, P.L[2], 0), cz), wrapped_sq(P, 2, r.z, cz),
                        wrapped_sq(P, 2, img_coord(r.z, P.L[2], 2), cz)};
  unsigned pass = 0;
#pragma unroll
  for (int ix = 0; ix < 3; ++ix) {
#pragma unroll
    for (int iy = 0; iy < 3; ++iy) {
      const double qxy = __dadd_rn(qx[ix], qy[iy]);
#pragma unroll
      for (int iz = 0; iz < 3; ++iz)
        pass |= (__dadd_rn(qxy, qz[iz]) >= thr ? 1u : 0u) << (9 * ix + 3 * iy + iz);
    }
  }
  return pass;
}

template <bool kMixed>
__device__ __forceinline__ void p2p_images(const OvParams& P, unsigned mask, d3 r, d3 r1, d3 r2,
                                           int id, int fw, int skip, double near2, d3& nl, d3& im,
                                           unsigned& n_p2p) {
  if (fw == -1) return;
  if (id == skip || fw == skip) mask &= ~(1u << kPrimary);
  n_p2p += __popc(mask);
  const d3 ds = r2 - r1;
  const double ds2 = dot3(ds, ds);
  const double far2 = fmax(16.0 * ds2, near2);
  const float dsx = (float)ds.x, dsy = (float)ds.y, dsz = (float)ds.z;
  const float f4 = (float)P.f4pi;
  float fx = 0, fy = 0, fz = 0;
  // one image per iteration, rolled: a single copy of each formula
#pragma unroll 1
  while (mask) {
    const int c = __ffs(mask) - 1;
    mask &= mask - 1;
    const int ix = (c * 57) >> 9, rem = c - 9 * ix, iy = (rem * 11) >> 5, iz = rem - 3 * iy;
    const d3 t = mk3(img_coord(r.x, P.L[0], ix), img_coord(r.y, P.L[1], iy), img_coord(r.z, P.L[2], iz));
    if (kMixed) {
      const d3 R = r1 - t;
      const double R2 = dot3(R, R);
      float vx, vy, vz;
      if (R2 >= far2 && ds2 > 0 &&
          seg_vel32(f4, (float)R.x, (float)R.y, (float)R.z, dsx, dsy, dsz, vx, vy, vz)) {
        fx += vx; fy += vy; fz += vz;
        continue;
      }
      // the mixed form keeps one sum for the tangle and its images
      nl = nl + seg64_at(P.f4pi, r1, r2, t);
      continue;
    }
    // the reference's formula with Newton-refined reciprocals (its own
    // operations near the cut-offs), as the FP64 direct sum
    const d3 v = seg_vel64_nr(P.f4pi, r1, r2, ds, t);
    if (c == kPrimary) nl = nl + v;
    else im = im + v;
  }
  if (kMixed) nl = nl + mk3(fx, fy, fz);
}

// Mixed form of one segment r1 -> r2 at every image in `mask` with many
// images: the images' offsets R = r1 - (r - L s) per axis and shift are
// formed in FP64 and rounded once, and two (x, y) image columns share each
// packed FP32 pair (columns 2g and 2g + 1, their three z images one after
// the other), as in cell_mixed.  Per image, with d = r2 - r1, a = |R|,
// b = |R + d|, u = 1/(ab), w = u / (1 + R.(R + d) u):
//   v = kappa/4pi (1/a + 1/b) w (R x d),   1 - cos = |R x d|^2 u w
// (the reference's segment formula, src/tangle.c:486-517, and its
// colinearity cut-off, zero inside it).  R x d, R.d and |R|^2 share their
// x and y parts along a column.  Images nearer than the far radius, or
// within 2.5e-3 of the cut-off, take the FP64 formula afterwards.  The skip
// rule (calculate_vs_shift, src/tangle.c:567-569) drops the tangle's own
// image for the target's own segments.
__device__ __forceinline__ void p2p_mixed_columns(const OvParams& P, unsigned mask, d3 r, d3 r1, d3 r2,
                                                  int id, int fw, int skip, double near2, d3& nl,
                                                  unsigned& n_p2p) {
  if (fw == -1) return;
  if (id == skip || fw == skip) mask &= ~(1u << kPrimary);
  n_p2p += __popc(mask);
  const d3 ds = r2 - r1;
  const double ds2 = dot3(ds, ds);
  const float far2 = (float)fmax(16.0 * ds2, near2);
  const float dx = (float)ds.x, dy = (float)ds.y, dz = (float)ds.z;
  const f2 Dx = f2_splat(dx), Dz = f2_splat(dz), nDy = f2_splat(-dy);
  const f2 D2 = f2_splat(fmaf(dx, dx, fmaf(dy, dy, dz * dz)));
  const f2 one = f2_splat(1.0f), two = f2_splat(2.0f);
  // FP32 copies of r1 - (r - L s) per axis and shift
  const float Fx[3] = {(float)__dsub_rn(r1.x, img_coord(r.x, P.L[0], 0)), (float)__dsub_rn(r1.x, r.x),
                       (float)__dsub_rn(r1.x, img_coord(r.x, P.L[0], 2))};
  const float Fy[3] = {(float)__dsub_rn(r1.y, img_coord(r.y, P.L[1], 0)), (float)__dsub_rn(r1.y, r.y),
                       (float)__dsub_rn(r1.y, img_coord(r.y, P.L[1], 2))};
  const float Fz[3] = {(float)__dsub_rn(r1.z, img_coord(r.z, P.L[2], 0)), (float)__dsub_rn(r1.z, r.z),
                       (float)__dsub_rn(r1.z, img_coord(r.z, P.L[2], 2))};
  f2 bx = f2_splat(0.f), by = bx, bz = bx;
  unsigned special = 0;   // images left to the FP64 formula
#pragma unroll
  for (int grp = 0; grp < 5; ++grp) {
    const int xa = 2 * grp, xb = grp < 4 ? xa + 1 : xa;
    const unsigned bits_a = (mask >> (3 * xa)) & 7u;
    const unsigned bits_b = grp < 4 ? (mask >> (3 * xb)) & 7u : 0u;
    if (!(bits_a | bits_b)) continue;
    const int ixa = (xa * 11) >> 5, iya = xa - 3 * ixa;
    const int ixb = (xb * 11) >> 5, iyb = xb - 3 * ixb;
    const f2 X = f2_pack(sel3f(ixa, Fx[0], Fx[1], Fx[2]), sel3f(ixb, Fx[0], Fx[1], Fx[2]));
    const f2 Y = f2_pack(sel3f(iya, Fy[0], Fy[1], Fy[2]), sel3f(iyb, Fy[0], Fy[1], Fy[2]));
    const f2 XY2 = f2_fma(X, X, Y * Y);
    const f2 XYd = f2_fma(X, Dx, Y * f2_splat(dy));
    const f2 Ydz = Y * Dz, mXdz = X * f2_splat(-dz);
    const f2 Cz = f2_fma(X, f2_splat(dy), Y * f2_splat(-dx));
    const f2 Cz2 = Cz * Cz;
#pragma unroll
    for (int iz = 0; iz < 3; ++iz) {
      const f2 Zs = f2_splat(Fz[iz]);
      const f2 R2 = f2_fma(Zs, Zs, XY2);
      const f2 Rd = f2_fma(Zs, Dz, XYd);
      const f2 Q2 = f2_fma(two, Rd, R2 + D2);
      const f2 ia = f2_rsqrt(R2), ib = f2_rsqrt(Q2);
      const f2 u = ia * ib;
      const f2 w = u * f2_rcp(f2_fma(R2 + Rd, u, one));
      const f2 s = (ia + ib) * w;
      const f2 Cx = f2_fma(Zs, nDy, Ydz);
      const f2 Cy = f2_fma(Zs, Dx, mXdz);
      const f2 tc = f2_fma(Cy, Cy, f2_fma(Cx, Cx, Cz2)) * (u * w);   // 1 - cos
      float tc0, tc1, r20, r21, s0, s1;
      f2_unpack(tc, tc0, tc1);
      f2_unpack(R2, r20, r21);
      f2_unpack(s, s0, s1);
      const bool in0 = (bits_a >> iz) & 1u, in1 = (bits_b >> iz) & 1u;
      const bool far0 = r20 >= far2, far1 = r21 >= far2;
      const bool ok0 = in0 && far0 && tc0 > kColHi, ok1 = in1 && far1 && tc1 > kColHi;
      // colinear (zero), masked-out and FP64 images add nothing here
      const f2 sk = f2_pack(ok0 ? s0 : 0.f, ok1 ? s1 : 0.f);
      bx = f2_fma(Cx, sk, bx);
      by = f2_fma(Cy, sk, by);
      bz = f2_fma(Cz, sk, bz);
      if (in0 && !ok0 && !(far0 && tc0 < kColLo)) special |= 1u << (3 * xa + iz);
      if (in1 && !ok1 && !(far1 && tc1 < kColLo)) special |= 1u << (3 * xb + iz);
    }
  }
  float lo, hi;
  const float f4 = (float)P.f4pi;
  f2_unpack(bx, lo, hi);
  const float fx = f4 * (lo + hi);
  f2_unpack(by, lo, hi);
  const float fy = f4 * (lo + hi);
  f2_unpack(bz, lo, hi);
  const float fz = f4 * (lo + hi);
  nl = nl + mk3(fx, fy, fz);
#pragma unroll 1
  while (special) {
    const int c = __ffs(special) - 1;
    special &= special - 1;
    const int ix = (c * 57) >> 9, rem = c - 9 * ix, iy = (rem * 11) >> 5, iz = rem - 3 * iy;
    nl = nl + seg64_at(P.f4pi, r1, r2,
                       mk3(img_coord(r.x, P.L[0], ix), img_coord(r.y, P.L[1], iy), img_coord(r.z, P.L[2], iz)));
  }
}

// images at which a segment is evaluated by columns rather than one by one
constexpr int kColumnImages = 8;

// Mixed form of one accepted cell at every image in `pass` (a 27-bit mask
// of the combos 9 (sx+1) + 3 (sy+1) + (sz+1)): FP32 expansions from the FP32
// moments at R = r - L s - com formed in FP64 and rounded once, summed in
// factored form and added to nl; images within the near radius in FP64
// (expansion64_at, added to nl as they come).  m21 is the FP32 m21 moment
// (the cell header's first word), thr the cell's opening threshold, dc the
// opening test's FP64 difference com - r.
__device__ __forceinline__ void cell_mixed(const OvParams& P, const Cell* cp, float m21, double cx, double cy,
                                           double cz, double thr, d3 r, d3 dc, unsigned pass, double near2,
                                           d3& nl) {
  const float2 q0f = *reinterpret_cast<const float2*>(&cp->f_g[0]);
  const float2 q1f = *reinterpret_cast<const float2*>(&cp->f_g[2]);
  const float2 q2f = *reinterpret_cast<const float2*>(&cp->f_m12);
  const float g0 = q0f.x, g1 = q0f.y, g2 = q1f.x, m02 = q1f.y, m12 = q2f.x, m22 = q2f.y;
  float ax, ay, az;
  {
    // FP32 copies of the FP64-formed offsets r - L s - com per axis and shift
    const float Fx[3] = {(float)__dsub_rn(img_coord(r.x, P.L[0], 0), cx),
                         -(float)dc.x,
                         (float)__dsub_rn(img_coord(r.x, P.L[0], 2), cx)};
    const float Fy[3] = {(float)__dsub_rn(img_coord(r.y, P.L[1], 0), cy),
                         -(float)dc.y,
                         (float)__dsub_rn(img_coord(r.y, P.L[1], 2), cy)};
    const float Fz[3] = {(float)__dsub_rn(img_coord(r.z, P.L[2], 0), cz),
                         -(float)dc.z,
                         (float)__dsub_rn(img_coord(r.z, P.L[2], 2), cz)};
    // an accepting image has |R|^2 >= its wrapped squared distance >=
    // thr, so a cell whose thr reaches the near radius needs no test
    const bool test_near = thr < near2;
    const float fnear2 = (float)near2;
    // two (x, y) columns per packed FP32 pair: columns 2g and 2g + 1
    // (the last group has column 8 only), their three z images
    // evaluated side by side (independent chains).  The 27 image
    // terms are summed in factored form: with i3 = |R|^-3 and
    // i5 = R_z |R|^-5 per image, the reference's
    // ((g + m R_z/|R|^2) x R + (m21, 0, 0)) i3 summed over the images
    // is g x P + m x Q + (m21 S, 0, 0), P = sum i3 R, Q = sum i5 R,
    // S = sum i3; since R_x and R_y are constant along a column,
    // P_x, P_y, Q_x, Q_y take each column's sums of i3 and i5 once.
    f2 px = f2_splat(0.f), py = px, pz = px, qx = px, qy = px, qz = px, sv = px;
    // All 27 images accept (the usual case: the wrapped opening test
    // treats every image point like the target) and none is near:
    // no per-image masks or near-field tests.  An image shifted
    // along an axis has |R|^2 >= that axis offset squared (FP32
    // rounding of sums of non-negative terms is monotonic), so when
    // every shifted offset and the target's own |R|^2 reach the near
    // radius, no image takes the FP64 path.
    bool all_far = pass == kAllImages;
    if (all_far && test_near) {
      const float X = Fx[1], Y = Fy[1], Z = Fz[1];
      all_far = fmaf(Z, Z, fmaf(X, X, Y * Y)) >= fnear2 && Fx[0] * Fx[0] >= fnear2 &&
                Fx[2] * Fx[2] >= fnear2 && Fy[0] * Fy[0] >= fnear2 && Fy[2] * Fy[2] >= fnear2 &&
                Fz[0] * Fz[0] >= fnear2 && Fz[2] * Fz[2] >= fnear2;
    }
    if (all_far) {
      // unrolled: the column offsets are chosen at compile time
#pragma unroll
      for (int grp = 0; grp < 5; ++grp) {
        const int xa = 2 * grp, xb = grp < 4 ? xa + 1 : xa;
        const int ixa = (xa * 11) >> 5, iya = xa - 3 * ixa;
        const int ixb = (xb * 11) >> 5, iyb = xb - 3 * ixb;
        const float Xa = sel3f(ixa, Fx[0], Fx[1], Fx[2]), Xb = sel3f(ixb, Fx[0], Fx[1], Fx[2]);
        const float Ya = sel3f(iya, Fy[0], Fy[1], Fy[2]), Yb = sel3f(iyb, Fy[0], Fy[1], Fy[2]);
        const f2 X = f2_pack(Xa, Xb), Y = f2_pack(Ya, Yb);
        const f2 XY2 = f2_fma(X, X, Y * Y);
        // the last group holds column 8 twice: its second half is dropped
        const f2 keep = f2_pack(1.f, grp < 4 ? 1.f : 0.f);
        f2 c3 = f2_splat(0.f), c5 = c3;
#pragma unroll
        for (int iz = 0; iz < 3; ++iz) {
          const f2 Zs = f2_splat(Fz[iz]);
          f2 inv = f2_rsqrt(f2_fma(Zs, Zs, XY2));
          if (grp == 4) inv = inv * keep;
          const f2 inv2 = inv * inv;
          const f2 i3 = inv2 * inv;
          const f2 i5 = (i3 * inv2) * Zs;
          c3 = c3 + i3;
          c5 = c5 + i5;
          pz = f2_fma(i3, Zs, pz);
          qz = f2_fma(i5, Zs, qz);
        }
        px = f2_fma(c3, X, px);
        py = f2_fma(c3, Y, py);
        qx = f2_fma(c5, X, qx);
        qy = f2_fma(c5, Y, qy);
        sv = sv + c3;
      }
    } else {
#pragma unroll 1
    for (int grp = 0; grp < 5; ++grp) {
      const int xa = 2 * grp, xb = grp < 4 ? xa + 1 : xa;
      const unsigned bits_a = (pass >> (3 * xa)) & 7u;
      const unsigned bits_b = grp < 4 ? (pass >> (3 * xb)) & 7u : 0u;
      if (!(bits_a | bits_b)) continue;
      const int ixa = (xa * 11) >> 5, iya = xa - 3 * ixa;
      const int ixb = (xb * 11) >> 5, iyb = xb - 3 * ixb;
      const float Xa = sel3f(ixa, Fx[0], Fx[1], Fx[2]), Xb = sel3f(ixb, Fx[0], Fx[1], Fx[2]);
      const float Ya = sel3f(iya, Fy[0], Fy[1], Fy[2]), Yb = sel3f(iyb, Fy[0], Fy[1], Fy[2]);
      const f2 X = f2_pack(Xa, Xb), Y = f2_pack(Ya, Yb);
      const f2 XY2 = f2_fma(X, X, Y * Y);
      float xy2a, xy2b;
      f2_unpack(XY2, xy2a, xy2b);
      // no z image of a column is nearer than its (x, y) distance
      const bool near_a = test_near && xy2a < fnear2, near_b = test_near && xy2b < fnear2;
      f2 c3 = f2_splat(0.f), c5 = c3;
#pragma unroll
      for (int iz = 0; iz < 3; ++iz) {
        const float Z = Fz[iz];
        const f2 Zs = f2_splat(Z);
        const f2 R2 = f2_fma(Zs, Zs, XY2);
        float r2a, r2b;
        f2_unpack(R2, r2a, r2b);
        bool on_a = (bits_a >> iz) & 1u, on_b = (bits_b >> iz) & 1u;
        if ((on_a && near_a) || (on_b && near_b)) {
          // near field: FP64 expansion from the FP64 offsets
          if (on_a && near_a && r2a < fnear2) {
            nl = nl + expansion64_at(cp, mk3(__dsub_rn(img_coord(r.x, P.L[0], ixa), cx),
                                             __dsub_rn(img_coord(r.y, P.L[1], iya), cy),
                                             __dsub_rn(img_coord(r.z, P.L[2], iz), cz)));
            on_a = false;
          }
          if (on_b && near_b && r2b < fnear2) {
            nl = nl + expansion64_at(cp, mk3(__dsub_rn(img_coord(r.x, P.L[0], ixb), cx),
                                             __dsub_rn(img_coord(r.y, P.L[1], iyb), cy),
                                             __dsub_rn(img_coord(r.z, P.L[2], iz), cz)));
            on_b = false;
          }
        }
        // images not evaluated here contribute exact zeros
        const f2 inv = f2_pack(on_a ? rsqrt_approx(r2a) : 0.f, on_b ? rsqrt_approx(r2b) : 0.f);
        const f2 inv2 = inv * inv;
        const f2 i3 = inv2 * inv;
        const f2 i5 = (i3 * inv2) * Zs;
        c3 = c3 + i3;
        c5 = c5 + i5;
        pz = f2_fma(i3, Zs, pz);
        qz = f2_fma(i5, Zs, qz);
      }
      px = f2_fma(c3, X, px);
      py = f2_fma(c3, Y, py);
      qx = f2_fma(c5, X, qx);
      qy = f2_fma(c5, Y, qy);
      sv = sv + c3;
    }
    }
    float a0, a1;
    f2_unpack(px, a0, a1);
    const float Px = a0 + a1;
    f2_unpack(py, a0, a1);
    const float Py = a0 + a1;
    f2_unpack(pz, a0, a1);
    const float Pz = a0 + a1;
    f2_unpack(qx, a0, a1);
    const float Qx = a0 + a1;
    f2_unpack(qy, a0, a1);
    const float Qy = a0 + a1;
    f2_unpack(qz, a0, a1);
    const float Qz = a0 + a1;
    f2_unpack(sv, a0, a1);
    const float S = a0 + a1;
    // g x P + m x Q + (m21 S, 0, 0), m = (m02, m12, m22)
    ax = fmaf(g1, Pz, fmaf(-g2, Py, fmaf(m12, Qz, fmaf(-m22, Qy, m21 * S))));
    ay = fmaf(g2, Px, fmaf(-g0, Pz, fmaf(m22, Qx, -m02 * Qz)));
    az = fmaf(g0, Py, fmaf(-g1, Px, fmaf(m02, Qy, -m12 * Qx)));
  }
  // the mixed form keeps one sum for the tangle and its images
  nl = nl + mk3(ax, ay, az);
}

// FP64 form of one accepted cell at every image in `pass`: the reference's
// expansion (src/octree.c:303-328) at R = r - L s - com.  The tangle's own
// image goes into nl as one evaluation; the other images are summed in
// factored form into im, as in cell_mixed: with i3 = |R|^-3 and
// i5 = R_z |R|^-5 per image, the sum of ((g + m R_z/|R|^2) x R + (m21, 0, 0)) i3
// is g x P + m x Q + (m21 S, 0, 0), P = sum i3 R, Q = sum i5 R, S = sum i3.
__device__ __forceinline__ void cell_fp64(const OvParams& P, const Cell* cp, double cx, double cy, double cz, d3 r,
                                          unsigned pass, d3& nl, d3& im) {
  const double g[3] = {cp->y[0], cp->y[1], cp->y[2]};
  const double mm[4] = {cp->m[0], cp->m[1], cp->m[2], cp->m[3]};
  const double Rz[3] = {__dsub_rn(img_coord(r.z, P.L[2], 0), cz), __dsub_rn(r.z, cz),
                        __dsub_rn(img_coord(r.z, P.L[2], 2), cz)};
  if (pass & (1u << kPrimary))
    nl = nl + expansion64(g, mm, mk3(__dsub_rn(r.x, cx), __dsub_rn(r.y, cy), Rz[1]));
  const unsigned rest = pass & ~(1u << kPrimary);
  if (!rest) return;
  double px = 0, py = 0, pz = 0, qx = 0, qy = 0, qz = 0, sv = 0;
#pragma unroll
  for (int xy = 0; xy < 9; ++xy) {
    const unsigned bits = (rest >> (3 * xy)) & 7u;
    if (!bits) continue;
    const int ix = (xy * 11) >> 5, iy = xy - 3 * ix;
    const double X = __dsub_rn(img_coord(r.x, P.L[0], ix), cx);
    const double Y = __dsub_rn(img_coord(r.y, P.L[1], iy), cy);
    const double XY2 = fma(X, X, Y * Y);
    double c3 = 0, c5 = 0;
#pragma unroll
    for (int iz = 0; iz < 3; ++iz) {
      if (!((bits >> iz) & 1u)) continue;
      const double Z = Rz[iz];
      const double inv = rsqrt(fma(Z, Z, XY2));
      const double inv2 = inv * inv;
      const double i3 = inv2 * inv;
      const double i5 = (i3 * inv2) * Z;
      c3 += i3;
      c5 += i5;
      pz = fma(i3, Z, pz);
      qz = fma(i5, Z, qz);
    }
    px = fma(c3, X, px);
    py = fma(c3, Y, py);
    qx = fma(c5, X, qx);
    qy = fma(c5, Y, qy);
    sv += c3;
  }
  // g x P + m x Q + (m21 S, 0, 0), m = (m02, m12, m22)
  const double m21 = mm[0], m02 = mm[1], m12 = mm[2], m22 = mm[3];
  im = im + mk3(fma(g[1], pz, fma(-g[2], py, fma(m12, qz, fma(-m22, qy, m21 * sv)))),
                fma(g[2], px, fma(-g[0], pz, fma(m22, qx, -m02 * qz))),
                fma(g[0], py, fma(-g[1], px, fma(m02, qy, -m12 * qx))));
}

// resident blocks per SM the register allocation must allow, measured at
// 1M points, ms per launch:
//   mixed 47.6 / 40.6 / 43.8 / 44.8 for 3 / 4 / 5 / 6 blocks (136 and 128
//   registers without spills, 96 registers and 56 bytes spilled, 80
//   registers and 272 bytes spilled)
//   FP64 87.6 / 79.8 / 78.5 for 4 / 5 / 6 blocks (110 registers without
//   spills, 96 registers and 48 bytes spilled, 80 registers and 88 bytes
//   spilled)
#ifndef OV_WALK_MULTI_MIN_BLOCKS_MIXED
#define OV_WALK_MULTI_MIN_BLOCKS_MIXED 4
#endif
#ifndef OV_WALK_MULTI_MIN_BLOCKS_FP64
#define OV_WALK_MULTI_MIN_BLOCKS_FP64 6
#endif

template <bool kMixed>
__global__ void __launch_bounds__(kMultiWarps * 32, kMixed ? OV_WALK_MULTI_MIN_BLOCKS_MIXED
                                                           : OV_WALK_MULTI_MIN_BLOCKS_FP64)
    k_walk_multi(
    OvParams P, TreeView T, const int* __restrict__ order, const int2* __restrict__ status,
    const double* __restrict__ pos, int n_t, unsigned combos, ImageShortcut S, double near2,
    double* v_nl, double* v_img, unsigned long long* counters, const int* __restrict__ warp_perm,
    unsigned* __restrict__ warp_cost) {
  __shared__ unsigned sh_mask[kMultiWarps][kLevelSlots][32];
  const unsigned FULL = 0xffffffffu;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long t_start = clock64();
  const int slot = blockIdx.x * kMultiWarps + warp;
  if (slot * 32 >= n_t) return;   // whole warp out of range
  // the group of 32 consecutive targets this warp takes: launch slot
  // `slot` runs group warp_perm[slot] (the groups by decreasing time in the
  // previous evaluation), or group `slot`
  const int gw = warp_perm ? warp_perm[slot] : slot;
  const int i = gw * 32 + lane;
  const int k = i < n_t ? (order ? order[i] : i) : -1;
  const bool live = k >= 0 && status[k].x != OV_PINNED && status[k].x != OV_EMPTY;
  const d3 r = live ? ld3(pos, k) : mk3(0, 0, 0);
  // the shortcuts' bound on rounding holds for targets within a quarter box
  // of the box (a node further out takes every decision in full)
  bool sane = S.on;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double v = a == 0 ? r.x : (a == 1 ? r.y : r.z);
    sane = sane && v >= P.lo[a] - 0.25 * P.L[a] && v <= P.hi[a] + 0.25 * P.L[a];
  }
  unsigned* lvl_mask = &sh_mask[warp][0][lane];   // level l at lvl_mask[32 l]
  lvl_mask[0] = combos;
  d3 nl = mk3(0, 0, 0), im = mk3(0, 0, 0);
  unsigned n_p2p = 0, n_far = 0, n_iter = 0;
  int next = live ? 0 : T.n_cells;
  __syncwarp();
  for (;;) {
    const int q = (int)__reduce_min_sync(FULL, (unsigned)next);
    if (q >= T.n_cells) break;
    const Cell* cp = T.cells + q;
    if (lane == 0 && q + 1 < T.n_cells) prefetch_l1(cp + 1);
    const int4 h = *reinterpret_cast<const int4*>(cp);
    const double2 t0 = *reinterpret_cast<const double2*>(&cp->thr);
    const double2 t1 = *reinterpret_cast<const double2*>(&cp->x[1]);
    const int kind = cell_kind(h.w);
    if (lane == 1 && h.z < T.n_cells) prefetch_l1(T.cells + h.z);
    unsigned p2p_mask = 0;   // images summing this cell's node range directly
    if (next == q) {
      const unsigned m = lvl_mask[32 * cell_ltop(h.w)];
      unsigned open = 0;
      if (kind == CELL_LEAF1) {
        if (kMixed && __popc(m) >= kColumnImages)
          p2p_mixed_columns(P, m, r, mk3(t0.y, t1.x, t1.y), mk3(cp->y[0], cp->y[1], cp->y[2]), h.x, h.y, k,
                            near2, nl, n_p2p);
        else
          p2p_images<kMixed>(P, m, r, mk3(t0.y, t1.x, t1.y), mk3(cp->y[0], cp->y[1], cp->y[2]), h.x,
                             h.y, k, near2, nl, im, n_p2p);
      } else if (kind == CELL_LEAFN) {
        p2p_mask = m;
      } else {
        // opening test per image (octree_get_vs, src/octree.c:284-296)
        const double cx = t0.y, cy = t1.x, cz = t1.y;
        // Per axis, an image point's exact wrapped distance to the centre
        // of mass is at least the target's, and equal to it when the
        // target's unwrapped difference c - r is below half a box (the
        // image's single wrap then undoes its shift).  The cell's margin E
        // (mac_margin) bounds the FP64 rounding of every image's squared
        // distance, so when the target's q0 passes by E every image passes,
        // and when q0 fails by E with no axis near half a box every image
        // fails.  Otherwise (and at the root, whose centre of mass may lie
        // outside the box) all decisions are taken in full.
        unsigned pass;
        // The reference wraps an axis when c - r lies outside [-L/2, L/2];
        // where no axis wraps its squared distance is that of c - r itself
        // (fl(r - c) = -fl(c - r)), bit for bit.
        const double dx = __dsub_rn(cx, r.x), dy = __dsub_rn(cy, r.y), dz = __dsub_rn(cz, r.z);
        double q0;
        if (fabs(dx) <= S.half[0] && fabs(dy) <= S.half[1] && fabs(dz) <= S.half[2])
          q0 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
        else
          q0 = __dadd_rn(__dadd_rn(wrapped_sq(P, 0, r.x, cx), wrapped_sq(P, 1, r.y, cy)), wrapped_sq(P, 2, r.z, cz));
        const double E = (double)__int_as_float(h.y);
        const bool shortcut = sane && q > 0;
        if (shortcut && q0 >= t0.x + E) {
          pass = m;
        } else if (shortcut && q0 < t0.x - E && fabs(dx) <= S.hw[0] && fabs(dy) <= S.hw[1] &&
                   fabs(dz) <= S.hw[2]) {
          pass = 0;
        } else {
          // q0 is the target's own decision in mac_exact's operations; the
          // other images still open here are few below the top levels, so
          // they are decided one by one unless there are many
          pass = q0 >= t0.x ? (1u << kPrimary) : 0u;
          unsigned rest = m & ~(1u << kPrimary);
          if (__popc(rest) > kFewImages) {
            pass |= mac_exact(P, r, cx, cy, cz, t0.x) & rest;
          } else {
            while (rest) {
              const int c = __ffs(rest) - 1;
              rest &= rest - 1;
              const int ix = (c * 57) >> 9, rem = c - 9 * ix, iy = (rem * 11) >> 5, iz = rem - 3 * iy;
              const double q = __dadd_rn(__dadd_rn(wrapped_sq(P, 0, img_coord(r.x, P.L[0], ix), cx),
                                                   wrapped_sq(P, 1, img_coord(r.y, P.L[1], iy), cy)),
                                         wrapped_sq(P, 2, img_coord(r.z, P.L[2], iz), cz));
              if (q >= t0.x) pass |= 1u << c;
            }
          }
        }
        pass &= m;
        const unsigned fail = m & ~pass;
        if (kind == CELL_OPEN) open = fail;
        else if (kind == CELL_OPEN_P2P) p2p_mask = fail;
        if (pass) {
          n_far += __popc(pass);
          // expansion at every accepting image: R = r - L s - com, unwrapped
          if (kMixed) {
            cell_mixed(P, cp, __int_as_float(h.x), cx, cy, cz, t0.x, r, mk3(dx, dy, dz), pass, near2, nl);
          } else {
            cell_fp64(P, cp, cx, cy, cz, r, pass, nl, im);
          }
        }
      }
      if (open) lvl_mask[32 * (cell_lbot(h.w) + 1)] = open;
      // each lane's next cell strictly increases: the loop ends within n_cells
      next = open ? q + 1 : max(h.z, q + 1);
    }
    ++n_iter;
    // direct sums over a node range (grain leaves), shared by the warp
    if (__ballot_sync(FULL, p2p_mask != 0)) {
      const int2 rg = T.cell_range[q];
      const int end = min(rg.x + rg.y, T.n_nodes);
      for (int j = max(rg.x, 0); j < end; ++j) {
        const int2 id = T.nodeids[j];
        if (!p2p_mask) continue;
        const double* nd = T.nodes64 + 6 * (size_t)j;
        if (kMixed && __popc(p2p_mask) >= kColumnImages)
          p2p_mixed_columns(P, p2p_mask, r, mk3(nd[0], nd[1], nd[2]), mk3(nd[3], nd[4], nd[5]), id.x, id.y,
                            k, near2, nl, n_p2p);
        else
          p2p_images<kMixed>(P, p2p_mask, r, mk3(nd[0], nd[1], nd[2]), mk3(nd[3], nd[4], nd[5]), id.x,
                             id.y, k, near2, nl, im, n_p2p);
      }
    }
  }
  if (live) {
    st3(v_nl, k, nl);
    st3(v_img, k, im);
  }
  // counters: per-warp sums
  unsigned long long a = n_p2p, b = n_far;
  for (int off = 16; off > 0; off >>= 1) {
    a += __shfl_xor_sync(FULL, a, off);
    b += __shfl_xor_sync(FULL, b, off);
  }
  if (lane == 0) {
    atomicAdd(&counters[0], a);
    atomicAdd(&counters[1], b);
    atomicAdd(&counters[2], (unsigned long long)n_iter);
    // this group's time in SM cycles / 64, for the next evaluation's order
    if (warp_cost) warp_cost[gw] = (unsigned)min((clock64() - t_start) >> 6, 0xffffffffll);
  }
}


// All nodes: warp w handles sorted targets 32w .. 32w+31, every image.
// Targets in `order` (the tree's key order, so a warp's targets are close in
// space), or slot order when order is null.
template <bool kMixed>
__global__ void __launch_bounds__(128) k_walk_nodes(OvParams P, TreeView T, const int* __restrict__ order,
                                                    const int2* __restrict__ status,
                                                    const double* __restrict__ pos, int n_t,
                                                    double* v_nl, double* v_img,
                                                    unsigned long long* counters) {
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int i = gw * 32 + lane;
  if (gw * 32 >= n_t) return;   // whole warp out of range
  int k = i < n_t ? (order ? order[i] : i) : -1;
  bool live = k >= 0 && status[k].x != OV_PINNED && status[k].x != OV_EMPTY;
  d3 r = live ? ld3(pos, k) : mk3(0, 0, 0);
  unsigned long long n_p2p = 0, n_far = 0, n_iter = 0;
  d3 nl = warp_walk<kMixed>(P, T, r, live, k, true, P.theta, n_p2p, n_far, n_iter);
  d3 im = mk3(0, 0, 0);
  for (int j = 0; j < P.n_img; ++j) {
    d3 rp = live ? image_point(P, j, r) : r;
    d3 v = warp_walk<kMixed>(P, T, rp, live, -1, true, P.theta, n_p2p, n_far, n_iter);
    int face = P.img[j][3];
    if (face > -1) v = mirror_dir(v, face);
    im = im + v;
  }
  if (live) {
    st3(v_nl, k, nl);
    st3(v_img, k, im);
  }
  if (lane == 0) {
    atomicAdd(&counters[0], n_p2p);
    atomicAdd(&counters[1], n_far);
    atomicAdd(&counters[2], n_iter);
  }
}

// Arbitrary points (octree_get_vs at user points), optionally with images.
template <bool kMixed>
__global__ void __launch_bounds__(128) k_walk_points(OvParams P, TreeView T, const double* __restrict__ pts,
                                                     const int* __restrict__ skip, int npts,
                                                     int use_thr, double theta, double* out_nl,
                                                     double* out_img, unsigned long long* counters) {
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int i = gw * 32 + lane;
  if (gw * 32 >= npts) return;
  bool live = i < npts;
  d3 r = live ? ld3(pts, i) : mk3(0, 0, 0);
  int sk = (live && skip) ? skip[i] : -1;
  unsigned long long n_p2p = 0, n_far = 0, n_iter = 0;
  d3 v = warp_walk<kMixed>(P, T, r, live, sk, use_thr != 0, theta, n_p2p, n_far, n_iter);
  if (out_img) {
    d3 im = mk3(0, 0, 0);
    for (int j = 0; j < P.n_img; ++j) {
      d3 rp = live ? image_point(P, j, r) : r;
      d3 w = warp_walk<kMixed>(P, T, rp, live, -1, use_thr != 0, theta, n_p2p, n_far, n_iter);
      int face = P.img[j][3];
      if (face > -1) w = mirror_dir(w, face);
      im = im + w;
    }
    if (live) st3(out_img, i, im);
  }
  if (live) st3(out_nl, i, v);
  if (lane == 0) {
    atomicAdd(&counters[0], n_p2p);
    atomicAdd(&counters[1], n_far);
    atomicAdd(&counters[2], n_iter);
  }
}

TreeView view_of(OvTree* t) {
  TreeView v;
  v.cells = t->cells.as<Cell>();
  v.cell_lm = t->cell_lm.as<double>();
  v.cell_range = t->cell_range.as<int2>();
  v.nodes64 = t->nodes64.as<double>();
  v.nodeids = t->nodeids.as<int2>();
  v.n_cells = t->n_cells;
  v.n_nodes = t->n_nodes;
  return v;
}

}  // namespace

// Target list with the nin nodes inside the root box after the nd outside
// it, each of those alone in a warp (lane 0; -1 marks an empty lane).
constexpr int kMaxDropWarps = 1024;
static __global__ void k_drop_first(const int* __restrict__ perm, int nin, int nd, int* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int pad = 32 * nd;
  if (i >= pad + nin) return;
  out[i] = i < pad ? ((i & 31) == 0 ? perm[nin + (i >> 5)] : -1) : perm[i - pad];
}

// sort keys for the groups' order: decreasing time first
static __global__ void k_cost_keys(const unsigned* __restrict__ cost, int n, uint64_t* keys, int* vals) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  keys[i] = (uint64_t)(0xffffffffu - cost[i]);
  vals[i] = i;
}

static bool read_counters(ov_state_impl* s, OvTree* t) {
  unsigned long long c[3] = {0, 0, 0};
  OV_TRY_CUDA(cudaMemcpyAsync(c, t->counters.as<char>() + 64, sizeof(c), cudaMemcpyDeviceToHost,
                              s->stream));
  OV_TRY_CUDA(cudaStreamSynchronize(s->stream));
  OvStatsAcc& st = ov_stats_tls();
  st.interactions = (double)c[0];
  st.cell_interactions = (double)c[1];
  st.warp_iterations = (double)c[2];
  return true;
}

bool ov_tree_walk_nodes(ov_state_impl* s, OvTree* t, const double* pos, bool own_tree,
                        double* v_nl, double* v_img, int k0, int k_count) {
  unsigned long long* ctr = reinterpret_cast<unsigned long long*>(t->counters.as<char>() + 64);
  OV_TRY_CUDA(cudaMemsetAsync(ctr, 0, 24, s->stream));
  // a tree built from these positions: its key order; otherwise slot order
  const int* order = own_tree ? t->perm.as<int>() : nullptr;
  int n_t = own_tree ? t->n_nodes : s->n;
  if (n_t == 0 || t->n_cells == 0) {
    OV_TRY_CUDA(cudaMemsetAsync(v_nl, 0, sizeof(double) * 3 * s->n, s->stream));
    OV_TRY_CUDA(cudaMemsetAsync(v_img, 0, sizeof(double) * 3 * s->n, s->stream));
    return true;
  }
  // one rank's share: a contiguous range of the key order (each target's
  // walk depends only on its own position, so the range changes no result)
  int key_lo = 0;   // key position of order[0]
  if (own_tree && k_count >= 0) {
    const int lo = std::min(std::max(k0, 0), n_t);
    key_lo = lo;
    n_t = std::min(k_count, n_t - lo);
    order += lo;
    if (n_t <= 0) {
      cudaEventRecord(s->ev1, s->stream);
      cudaEventRecord(s->ev2, s->stream);
      return read_counters(s, t);
    }
  }
  // Nodes outside the root box take key digit 8 at level 1 and sort after
  // every other node, so they would share the last warps whatever their
  // positions.  A warp of targets scattered over the box's faces walks the
  // union of their trees, and as the last block it ran almost alone at the
  // end of the launch: 20 such nodes made a 1M-point walk 28% longer.  Each
  // gets a warp of its own at the front of the list instead (the other lanes
  // empty); the sums do not depend on the order.  In a rank's share of the
  // key order these nodes are the share's last ones.
  const int nd = own_tree ? std::max(0, std::min(n_t, key_lo + n_t - (t->n_nodes - t->n_drop_root))) : 0;
  if (nd > 0 && t->n_drop_root <= kMaxDropWarps) {
    const int nin = n_t - nd;
    const int m = 32 * nd + nin;
    if (!t->walk_order.reserve(sizeof(int) * (size_t)m)) return false;
    k_drop_first<<<(m + 255) / 256, 256, 0, s->stream>>>(order, nin, nd, t->walk_order.as<int>());
    OV_LAUNCHED();
    OV_TRY_CUDA(cudaGetLastError());
    order = t->walk_order.as<int>();
    n_t = m;
  }
  TreeView tv = view_of(t);
  OvParams P = t->P;
  // image table and precision of this call; geometry of the tree's build
  P.n_img = s->P.n_img;
  for (int j = 0; j < P.n_img; ++j)
    for (int c = 0; c < 4; ++c) P.img[j][c] = s->P.img[j][c];
  P.precision = s->P.precision;
  const bool mixed = s->P.precision == OV_PREC_MIXED;
  // images as a set of periodic shifts in {-1,0,1}^3 without mirrors or
  // repeats: one multi-image walk per target
  unsigned combos = 1u << 13;
  bool multi = true;
  for (int j = 0; j < P.n_img && multi; ++j) {
    const int* im = P.img[j];
    if (im[3] != -1 || im[0] < -1 || im[0] > 1 || im[1] < -1 || im[1] > 1 || im[2] < -1 ||
        im[2] > 1) {
      multi = false;
      break;
    }
    unsigned bit = 1u << (9 * (im[0] + 1) + 3 * (im[1] + 1) + (im[2] + 1));
    if (combos & bit) multi = false;
    combos |= bit;
  }
  const double near2 = s->P.near2;
  // shortcut parameters: see ImageShortcut and mac_margin (the rounding
  // allowance 8 u B with B the bound on magnitudes of mac_margin)
  ImageShortcut sc;
  {
    double B = 0;
    for (int a = 0; a < 3; ++a) B = std::max(B, std::fabs(P.lo[a]) + std::fabs(P.hi[a]));
    const double allowance = 8 * 0x1p-53 * 3.5 * B;
    sc.on = 1;
    for (int a = 0; a < 3; ++a) {
      bool shifted = false;
      for (int c = 0; c < kCombos; ++c) {
        const int sa = a == 0 ? c / 9 : (a == 1 ? (c / 3) % 3 : c % 3);
        if (((combos >> c) & 1u) && sa != 1) shifted = true;
      }
      if (shifted && !P.periodic[a]) sc.on = 0;
      sc.hw[a] = shifted ? 0.5 * P.L[a] - allowance : DBL_MAX;
      sc.half[a] = P.periodic[a] ? P.L[a] * 0.5 : DBL_MAX;
    }
  }
  cudaEventRecord(s->ev1, s->stream);
  if (multi) {
    int warps = (n_t + 31) / 32;
    int blocks = (warps + kMultiWarps - 1) / kMultiWarps;
    // Longest groups first: the launch runs the groups of 32 targets in the
    // order of their times in the previous walk of this tree (the same
    // regions of the key order, a few node moves apart), so the slow ones
    // do not start in the last wave.  The sums do not depend on the order.
    // A rank's share of a sharded evaluation is the same key range at every
    // evaluation, so its groups are ordered the same way.
    const bool timed = own_tree;
    const int* wperm = timed && t->n_perm_warps == warps ? t->wvals.as<int>() : nullptr;
    unsigned* wcost = nullptr;
    if (timed) {
      if (!t->warp_cost.reserve(sizeof(unsigned) * (size_t)warps)) return false;
      wcost = t->warp_cost.as<unsigned>();
    }
    if (mixed) {
      k_walk_multi<true><<<blocks, kMultiWarps * 32, 0, s->stream>>>(
          P, tv, order, s->status.as<int2>(), pos, n_t, combos, sc, near2, v_nl, v_img, ctr, wperm, wcost);
      OV_LAUNCHED();
    } else {
      k_walk_multi<false><<<blocks, kMultiWarps * 32, 0, s->stream>>>(
          P, tv, order, s->status.as<int2>(), pos, n_t, combos, sc, near2, v_nl, v_img, ctr, wperm, wcost);
      OV_LAUNCHED();
    }
    OV_TRY_CUDA(cudaGetLastError());
    cudaEventRecord(s->ev2, s->stream);
    if (timed) {
      // the order for the next walk (after the timed kernel)
      const size_t nw = (size_t)warps;
      if (!t->wkeys.reserve(sizeof(uint64_t) * nw) || !t->wkeys2.reserve(sizeof(uint64_t) * nw) ||
          !t->wvals.reserve(sizeof(int) * nw) || !t->wvals2.reserve(sizeof(int) * nw))
        return false;
      k_cost_keys<<<(warps + 255) / 256, 256, 0, s->stream>>>(wcost, warps, t->wkeys.as<uint64_t>(),
                                                                t->wvals.as<int>());
      OV_LAUNCHED();
      if (!ov_radix_sort_u64(t->wkeys.as<uint64_t>(), t->wvals.as<int>(), t->wkeys2.as<uint64_t>(),
                             t->wvals2.as<int>(), warps, t->whist, t->wscan, s->stream))
        return false;
      t->n_perm_warps = warps;
    }
    return read_counters(s, t);
  } else {
    int warps = (n_t + 31) / 32;
    int blocks = (warps * 32 + 127) / 128;
    if (mixed) {
      k_walk_nodes<true><<<blocks, 128, 0, s->stream>>>(P, tv, order, s->status.as<int2>(), pos, n_t,
                                                         v_nl, v_img, ctr);
      OV_LAUNCHED();
    } else {
      k_walk_nodes<false><<<blocks, 128, 0, s->stream>>>(P, tv, order, s->status.as<int2>(), pos, n_t,
                                                          v_nl, v_img, ctr);
      OV_LAUNCHED();
    }
  }
  OV_TRY_CUDA(cudaGetLastError());
  cudaEventRecord(s->ev2, s->stream);
  return read_counters(s, t);
}

bool ov_tree_walk_points(ov_state_impl* s, OvTree* t, int npts, const double* pts, const int* skip,
                         double theta, double* out_nl, double* out_img) {
  if (npts <= 0) return true;
  if (t->n_cells == 0) {
    OV_TRY_CUDA(cudaMemsetAsync(out_nl, 0, sizeof(double) * 3 * npts, s->stream));
    if (out_img) OV_TRY_CUDA(cudaMemsetAsync(out_img, 0, sizeof(double) * 3 * npts, s->stream));
    return true;
  }
  unsigned long long* ctr = reinterpret_cast<unsigned long long*>(t->counters.as<char>() + 64);
  OV_TRY_CUDA(cudaMemsetAsync(ctr, 0, 24, s->stream));
  int warps = (npts + 31) / 32;
  int blocks = (warps * 32 + 127) / 128;
  TreeView tv = view_of(t);
  OvParams P = t->P;
  P.n_img = s->P.n_img;
  for (int j = 0; j < P.n_img; ++j)
    for (int c = 0; c < 4; ++c) P.img[j][c] = s->P.img[j][c];
  int use_thr = theta == t->theta;
  if (s->P.precision == OV_PREC_MIXED) {
    k_walk_points<true><<<blocks, 128, 0, s->stream>>>(P, tv, pts, skip, npts, use_thr, theta,
                                                        out_nl, out_img, ctr);
    OV_LAUNCHED();
  }
  else {
    k_walk_points<false><<<blocks, 128, 0, s->stream>>>(P, tv, pts, skip, npts, use_thr, theta,
                                                         out_nl, out_img, ctr);
    OV_LAUNCHED();
  }
  OV_TRY_CUDA(cudaGetLastError());
  return read_counters(s, t);
}

// ---------------------------------------------------------------- shards
namespace {

__global__ void k_shard_pack(const int* __restrict__ perm, int k0, int count,
                             const double* __restrict__ v_nl, const double* __restrict__ v_img,
                             double* xbuf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int k = perm[k0 + i];
  double* o = xbuf + 6 * ((size_t)k0 + i);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    o[c] = v_nl[3 * (size_t)k + c];
    o[3 + c] = v_img[3 * (size_t)k + c];
  }
}

__global__ void k_shard_unpack(const int* __restrict__ perm, int n, const double* __restrict__ xbuf,
                               double* v_nl, double* v_img) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k = perm[i];
  const double* x = xbuf + 6 * (size_t)i;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    v_nl[3 * (size_t)k + c] = x[c];
    v_img[3 * (size_t)k + c] = x[3 + c];
  }
}

// the exchange buffer holds 6 doubles per key position of the tree
bool shard_fits(ov_state_impl* s, size_t xcap) {
  if (6 * (size_t)s->tree.n_nodes <= xcap) return true;
  ov_set_error(OV_ERR_INVALID, "tree of %d nodes beyond the exchange buffer (%zu doubles): call "
               "ov_state_shard after the upload", s->tree.n_nodes, xcap);
  return false;
}

}  // namespace

bool ov_shard_pack(ov_state_impl* s, int k0, int count, double* xbuf, size_t xcap) {
  if (!shard_fits(s, xcap)) return false;
  const int n = s->tree.n_nodes;
  k0 = std::min(std::max(k0, 0), n);
  count = std::min(count, n - k0);
  if (count <= 0) return true;
  k_shard_pack<<<(count + 255) / 256, 256, 0, s->stream>>>(s->tree.perm.as<int>(), k0, count,
                                                           s->v_nl.as<double>(), s->v_img.as<double>(), xbuf);
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  return true;
}

bool ov_shard_unpack(ov_state_impl* s, const double* xbuf, size_t xcap) {
  if (!shard_fits(s, xcap)) return false;
  const int n = s->tree.n_nodes;
  if (n <= 0) return true;
  k_shard_unpack<<<(n + 255) / 256, 256, 0, s->stream>>>(s->tree.perm.as<int>(), n, xbuf,
                                                         s->v_nl.as<double>(), s->v_img.as<double>());
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  return true;
}
