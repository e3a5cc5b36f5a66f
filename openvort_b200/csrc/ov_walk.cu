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
  const CellMeta* meta;
  const CellMom64* mom64;
  const CellMom32* mom32;
  const double* nodes64;   // per sorted node: r1, wrapped r2
  const int2* nodeids;     // per sorted node: slot, forward slot
  int n_cells;
  int n_nodes;
};

// squared distance from r to the cell's centre of mass after the reference's
// one-box wrap of the centre (seg_pwrap + segment_len, src/octree.c:286-287),
// with exactly its FP64 operations
__device__ __forceinline__ double mac_dist2(const OvParams& P, d3 r, const double* com) {
  double u[3];
  const double rr[3] = {r.x, r.y, r.z};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double c = com[a];
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
__device__ __forceinline__ d3 expansion64(const CellMom64& m, d3 R) {
  double R2 = dot3(R, R);
  double inv = 1.0 / sqrt(R2);
  double i3 = inv * inv * inv;
  double i5 = i3 * inv * inv;
  d3 g = mk3(m.gam[0], m.gam[1], m.gam[2]);
  d3 v = cross3(g, R) * i3;
  v.x += m.m21 * i3;
  d3 mv = mk3(m.m02 * R.z, m.m12 * R.z, m.m22 * R.z);
  return v + cross3(mv, R) * i5;
}

__device__ __forceinline__ void expansion32(const CellMom32& m, float Rx, float Ry, float Rz,
                                            float& vx, float& vy, float& vz) {
  float R2 = fmaf(Rx, Rx, fmaf(Ry, Ry, Rz * Rz));
  float inv = rsqrtf(R2);
  float i3 = inv * inv * inv;
  float i5 = i3 * inv * inv;
  float cx = m.gam[1] * Rz - m.gam[2] * Ry;
  float cy = m.gam[2] * Rx - m.gam[0] * Rz;
  float cz = m.gam[0] * Ry - m.gam[1] * Rx;
  float ax = m.m02 * Rz, ay = m.m12 * Rz, az = m.m22 * Rz;
  float qx = ay * Rz - az * Ry, qy = az * Rx - ax * Rz, qz = ax * Ry - ay * Rx;
  vx = fmaf(cx + m.m21, i3, qx * i5);
  vy = fmaf(cy, i3, qy * i5);
  vz = fmaf(cz, i3, qz * i5);
}

enum { ACT_NONE = 0, ACT_P2P = 1, ACT_FAR = 2, ACT_OPEN = 3 };

// One walk of one warp: lane targets rp (valid if `live`), skip rule `skip`.
// Returns the lane's sum; counts interactions.
template <bool kMixed>
__device__ d3 warp_walk(const OvParams& P, const TreeView& T, d3 rp, bool live, int skip,
                        bool use_thr, double theta, unsigned long long& n_p2p,
                        unsigned long long& n_far) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  int next = live ? 0 : T.n_cells;
  double ax = 0, ay = 0, az = 0;
  for (;;) {
    int q = __reduce_min_sync(FULL, (unsigned)next);
    if (q >= T.n_cells) break;
    const CellMeta m = T.meta[q];
    int act = ACT_NONE;
    if (next == q) {
      if (m.kind == CELL_LEAF) {
        act = ACT_P2P;
      } else {
        const double* com = T.mom64[q].com;
        double s = mac_dist2(P, rp, com);
        bool pass = use_thr ? (s >= m.thr)
                            : (s > 0 && __ddiv_rn(m.Lm, __dsqrt_rn(s)) < theta);
        if (pass) act = ACT_FAR;
        else if (m.kind == CELL_OPEN) act = ACT_OPEN;
        else if (m.kind == CELL_OPEN_P2P) act = ACT_P2P;
        else act = ACT_NONE;
      }
      // every lane's next cell strictly increases, so a walk ends within
      // n_cells iterations whatever the cell records hold
      next = (act == ACT_OPEN) ? q + 1 : max(m.skip, q + 1);
    }
    if (act == ACT_FAR) {
      if (kMixed) {
        const double* com = T.mom64[q].com;
        float Rx = (float)(rp.x - com[0]), Ry = (float)(rp.y - com[1]), Rz = (float)(rp.z - com[2]);
        float vx, vy, vz;
        expansion32(T.mom32[q], Rx, Ry, Rz, vx, vy, vz);
        ax += vx; ay += vy; az += vz;
      } else {
        const CellMom64 mm = T.mom64[q];
        d3 R = mk3(rp.x - mm.com[0], rp.y - mm.com[1], rp.z - mm.com[2]);
        d3 v = expansion64(mm, R);
        ax += v.x; ay += v.y; az += v.z;
      }
    }
    unsigned far_mask = __ballot_sync(FULL, act == ACT_FAR);
    unsigned p2p_mask = __ballot_sync(FULL, act == ACT_P2P);
    if (lane == 0) n_far += __popc(far_mask);
    if (p2p_mask) {
      const int end = min(m.start + m.count, T.n_nodes);
      if (lane == 0) n_p2p += (unsigned long long)__popc(p2p_mask) * m.count;
      for (int i = max(m.start, 0); i < end; ++i) {
        const int2 id = T.nodeids[i];
        if (act != ACT_P2P) continue;
        // skip rule of calculate_vs_shift (src/tangle.c:567-569)
        if (id.y == -1 || id.x == skip || id.y == skip) continue;
        const double* nd = T.nodes64 + 6 * (size_t)i;
        d3 r1 = mk3(nd[0], nd[1], nd[2]), r2 = mk3(nd[3], nd[4], nd[5]);
        if (kMixed) {
          d3 R = r1 - rp;
          d3 ds = r2 - r1;
          double R2 = dot3(R, R), ds2 = dot3(ds, ds);
          if (R2 >= 16.0 * ds2 && ds2 > 0) {
            float vx, vy, vz;
            seg_vel32((float)P.f4pi, (float)R.x, (float)R.y, (float)R.z, (float)ds.x, (float)ds.y,
                      (float)ds.z, vx, vy, vz);
            ax += vx; ay += vy; az += vz;
            continue;
          }
        }
        d3 v = seg_vel64(P.f4pi, r1, r2, rp);
        ax += v.x; ay += v.y; az += v.z;
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
  unsigned long long n_p2p = 0, n_far = 0;
  d3 nl = warp_walk<kMixed>(P, T, r, live, k, true, P.theta, n_p2p, n_far);
  d3 im = mk3(0, 0, 0);
  for (int j = 0; j < P.n_img; ++j) {
    d3 rp = live ? image_point(P, j, r) : r;
    d3 v = warp_walk<kMixed>(P, T, rp, live, -1, true, P.theta, n_p2p, n_far);
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
  unsigned long long n_p2p = 0, n_far = 0;
  d3 v = warp_walk<kMixed>(P, T, r, live, sk, use_thr != 0, theta, n_p2p, n_far);
  if (out_img) {
    d3 im = mk3(0, 0, 0);
    for (int j = 0; j < P.n_img; ++j) {
      d3 rp = live ? image_point(P, j, r) : r;
      d3 w = warp_walk<kMixed>(P, T, rp, live, -1, use_thr != 0, theta, n_p2p, n_far);
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
  }
}

TreeView view_of(OvTree* t) {
  TreeView v;
  v.meta = t->meta.as<CellMeta>();
  v.mom64 = t->mom64.as<CellMom64>();
  v.mom32 = t->mom32.as<CellMom32>();
  v.nodes64 = t->nodes64.as<double>();
  v.nodeids = t->nodeids.as<int2>();
  v.n_cells = t->n_cells;
  v.n_nodes = t->n_nodes;
  return v;
}

}  // namespace

static bool read_counters(ov_state_impl* s, OvTree* t) {
  unsigned long long c[2] = {0, 0};
  OV_TRY_CUDA(cudaMemcpyAsync(c, t->counters.as<char>() + 64, sizeof(c), cudaMemcpyDeviceToHost,
                              s->stream));
  OV_TRY_CUDA(cudaStreamSynchronize(s->stream));
  OvStatsAcc& st = ov_stats_tls();
  st.interactions = (double)c[0];
  st.cell_interactions = (double)c[1];
  return true;
}

bool ov_tree_walk_nodes(ov_state_impl* s, OvTree* t, const double* pos, bool own_tree,
                        double* v_nl, double* v_img) {
  unsigned long long* ctr = reinterpret_cast<unsigned long long*>(t->counters.as<char>() + 64);
  OV_TRY_CUDA(cudaMemsetAsync(ctr, 0, 16, s->stream));
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
  OV_TRY_CUDA(cudaMemsetAsync(ctr, 0, 16, s->stream));
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
