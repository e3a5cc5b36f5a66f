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

#include "ov_internal.h"

namespace {

struct TreeView {
  const Cell* cells;
  const double* cell_lm;   // max box side per cell (opening test at a user theta)
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
__device__ __forceinline__ d3 expansion64(const double* g, const double* m, d3 R) {
  double R2 = dot3(R, R);
  double inv = 1.0 / sqrt(R2);
  double i3 = inv * inv * inv;
  double i5 = i3 * inv * inv;
  d3 v = cross3(mk3(g[0], g[1], g[2]), R) * i3;
  v.x += m[0] * i3;
  d3 mv = mk3(m[1] * R.z, m[2] * R.z, m[3] * R.z);
  return v + cross3(mv, R) * i5;
}

__device__ __forceinline__ void expansion32(float g0, float g1, float g2, float m21, float m02,
                                            float m12, float m22, float Rx, float Ry, float Rz,
                                            float& vx, float& vy, float& vz) {
  float R2 = fmaf(Rx, Rx, fmaf(Ry, Ry, Rz * Rz));
  float inv = rsqrtf(R2);
  float i3 = inv * inv * inv;
  float i5 = i3 * inv * inv;
  float cx = g1 * Rz - g2 * Ry;
  float cy = g2 * Rx - g0 * Rz;
  float cz = g0 * Ry - g1 * Rx;
  float ax = m02 * Rz, ay = m12 * Rz, az = m22 * Rz;
  float qx = ay * Rz - az * Ry, qy = az * Rx - ax * Rz, qz = ax * Ry - ay * Rx;
  vx = fmaf(cx + m21, i3, qx * i5);
  vy = fmaf(cy, i3, qy * i5);
  vz = fmaf(cz, i3, qz * i5);
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
    if (R2 >= 16.0 * ds2 && ds2 > 0) {
      float vx, vy, vz;
      seg_vel32((float)P.f4pi, (float)R.x, (float)R.y, (float)R.z, (float)ds.x, (float)ds.y,
                (float)ds.z, vx, vy, vz);
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
    const int4 h = *reinterpret_cast<const int4*>(cp);           // a, b, skip|kind, f_m21
    const double2 t0 = *reinterpret_cast<const double2*>(&cp->thr);  // thr, x0
    const double2 t1 = *reinterpret_cast<const double2*>(&cp->x[1]); // x1, x2
    const int kind = (unsigned)h.z >> CELL_KIND_SHIFT;
    const int skp = h.z & CELL_SKIP_MASK;
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
        expansion32(f0.x, f0.y, f1.x, __int_as_float(h.w), f1.y, f2.x, f2.y, (float)(rp.x - t0.y),
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
      const int end = min(h.x + h.y, T.n_nodes);
      if (lane == 0) n_p2p += (unsigned long long)__popc(pn_mask) * h.y;
      for (int i = max(h.x, 0); i < end; ++i) {
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
  v.nodes64 = t->nodes64.as<double>();
  v.nodeids = t->nodeids.as<int2>();
  v.n_cells = t->n_cells;
  v.n_nodes = t->n_nodes;
  return v;
}

}  // namespace

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
                        double* v_nl, double* v_img) {
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
  int warps = (n_t + 31) / 32;
  int blocks = (warps * 32 + 127) / 128;
  TreeView tv = view_of(t);
  OvParams P = t->P;
  // image table and precision of this call; geometry of the tree's build
  P.n_img = s->P.n_img;
  for (int j = 0; j < P.n_img; ++j)
    for (int c = 0; c < 4; ++c) P.img[j][c] = s->P.img[j][c];
  cudaEventRecord(s->ev1, s->stream);
  if (s->P.precision == OV_PREC_MIXED) {
    k_walk_nodes<true><<<blocks, 128, 0, s->stream>>>(P, tv, order, s->status.as<int2>(), pos, n_t,
                                                       v_nl, v_img, ctr);
    OV_LAUNCHED();
  }
  else {
    k_walk_nodes<false><<<blocks, 128, 0, s->stream>>>(P, tv, order, s->status.as<int2>(), pos, n_t,
                                                        v_nl, v_img, ctr);
    OV_LAUNCHED();
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
