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
// FP64 form: the reference's formula and cut-offs (seg_vel64).
// Mixed form: sources staged as FP32 offsets from the block's first target
// (the subtraction done in FP64, rounded once); far segments (|R| >= 4|ds|)
// take the FP32 formula, near ones fall back to seg_vel64 from the FP64
// table; sums accumulate in FP64.
#include "ov_internal.h"

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
// explicit points.  Sources: all slots, or the list `only`.
__global__ void __launch_bounds__(kTB) k_direct64(OvParams P, SegTab S, int n_src, const int* only,
                                                  const double* __restrict__ tpos,
                                                  const int2* __restrict__ tstatus,
                                                  const int* __restrict__ tskip, int n_t,
                                                  double* __restrict__ part) {
  __shared__ double sh_r[kTS][6];
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
  for (int base = 0; base < n_src; base += kTS) {
    __syncthreads();
    for (int q = threadIdx.x; q < kTS; q += kTB) {
      int m = base + q;
      int id = -1, fw = -1;
      if (m < n_src) {
        id = only ? only[m] : m;
        fw = S.fwd[id];
        const double* src = S.r1r2 + 6 * id;
#pragma unroll
        for (int c = 0; c < 6; ++c) sh_r[q][c] = src[c];
      }
      sh_id[q][0] = id;
      sh_id[q][1] = fw;
    }
    __syncthreads();
    if (!act) continue;
    int cnt = min(kTS, n_src - base);
    for (int q = 0; q < cnt; ++q) {
      int id = sh_id[q][0], fw = sh_id[q][1];
      // skip rule of calculate_vs_shift (src/tangle.c:567-569)
      if (fw == -1 || id == skip || fw == skip) continue;
      d3 v = seg_vel64(f4pi, mk3(sh_r[q][0], sh_r[q][1], sh_r[q][2]),
                       mk3(sh_r[q][3], sh_r[q][4], sh_r[q][5]), r);
      ax += v.x; ay += v.y; az += v.z;
    }
  }
  if (act) {
    double* o = part + (size_t)j * 3 * n_t + 3 * (size_t)k;
    o[0] = ax; o[1] = ay; o[2] = az;
  } else if (k < n_t) {
    double* o = part + (size_t)j * 3 * n_t + 3 * (size_t)k;
    o[0] = 0; o[1] = 0; o[2] = 0;
  }
}

// Mixed form.  Segments closer than max(4 |ds|, the near radius) use the
// FP64 formula from the FP64 table.  Sources and targets are FP64 offsets from the block origin O
// (the block's first target's point for this image) split into two FP32
// parts, hi = fl32(p - O) and lo = fl32((p - O) - hi); R = (a_hi - t_hi) +
// (a_lo - t_lo) then carries ~2 FP32 ulps of |R| itself, however far the
// source and target are from O.
__global__ void __launch_bounds__(kTB) k_direct_mixed(OvParams P, SegTab S, int n_src,
                                                      const double* __restrict__ tpos,
                                                      const int2* __restrict__ tstatus,
                                                      const int* __restrict__ order, int n_t,
                                                      int stride, double* __restrict__ part) {
  __shared__ float4 sh_hi[kTS];   // r1 - O (hi part), w = 16 |ds|^2
  __shared__ float4 sh_lo[kTS];   // r1 - O (lo part)
  __shared__ float4 sh_d[kTS];    // ds
  __shared__ int sh_id[kTS][2];
  __shared__ double sh_O[3];
  const int j = blockIdx.y;
  const int i = blockIdx.x * kTB + threadIdx.x;   // position in `order`
  int k = i < n_t ? (order ? order[i] : i) : -1;
  bool act = k >= 0 && tstatus[k].x != OV_EMPTY && tstatus[k].x != OV_PINNED;
  d3 r = mk3(0, 0, 0);
  if (k >= 0) {
    r = ld3(tpos, k);
    if (j > 0) r = image_point(P, j - 1, r);
  }
  if (threadIdx.x == 0) {
    int k0 = order ? order[blockIdx.x * kTB] : blockIdx.x * kTB;
    d3 o = ld3(tpos, k0);
    if (j > 0) o = image_point(P, j - 1, o);
    sh_O[0] = o.x; sh_O[1] = o.y; sh_O[2] = o.z;
  }
  __syncthreads();
  const d3 O = mk3(sh_O[0], sh_O[1], sh_O[2]);
  const int skip = (j == 0) ? k : -1;
  const double ex = r.x - O.x, ey = r.y - O.y, ez = r.z - O.z;
  const float thx = (float)ex, thy = (float)ey, thz = (float)ez;
  const float tlx = (float)(ex - thx), tly = (float)(ey - thy), tlz = (float)(ez - thz);
  double ax = 0, ay = 0, az = 0;
  const float f4 = (float)P.f4pi;
  for (int base = 0; base < n_src; base += kTS) {
    __syncthreads();
    for (int q = threadIdx.x; q < kTS; q += kTB) {
      int m = base + q;
      int id = -1, fw = -1;
      float4 hi = make_float4(0, 0, 0, 0), lo = make_float4(0, 0, 0, 0), d = make_float4(0, 0, 0, 0);
      if (m < n_src) {
        id = order ? order[m] : m;
        fw = S.fwd[id];
        if (fw >= 0) {
          const double* src = S.r1r2 + 6 * id;
          double dx = src[3] - src[0], dy = src[4] - src[1], dz = src[5] - src[2];
          double px = src[0] - O.x, py = src[1] - O.y, pz = src[2] - O.z;
          float hx = (float)px, hy = (float)py, hz = (float)pz;
          // FP32 beyond max(4 |ds|, the near radius)
          hi = make_float4(hx, hy, hz, (float)fmax(16.0 * (dx * dx + dy * dy + dz * dz), P.near2));
          lo = make_float4((float)(px - hx), (float)(py - hy), (float)(pz - hz), 0.f);
          d = make_float4((float)dx, (float)dy, (float)dz, 0.f);
        }
      }
      sh_hi[q] = hi;
      sh_lo[q] = lo;
      sh_d[q] = d;
      sh_id[q][0] = id;
      sh_id[q][1] = fw;
    }
    __syncthreads();
    if (!act) continue;
    int cnt = min(kTS, n_src - base);
    // FP32 partial sums over 32 sources, each flushed into the FP64 sum
    for (int q0 = 0; q0 < cnt; q0 += 32) {
      float bx = 0, by = 0, bz = 0;
      int q1 = min(q0 + 32, cnt);
      for (int q = q0; q < q1; ++q) {
        const float4 a = sh_hi[q];
        const float4 l = sh_lo[q];
        const float4 d = sh_d[q];
        float Rx = (a.x - thx) + (l.x - tlx);
        float Ry = (a.y - thy) + (l.y - tly);
        float Rz = (a.z - thz) + (l.z - tlz);
        float R2 = fmaf(Rx, Rx, fmaf(Ry, Ry, Rz * Rz));
        const int id = sh_id[q][0], fw = sh_id[q][1];
        // skip rule of calculate_vs_shift (src/tangle.c:567-569) at any
        // distance: across a periodic face a neighbour's segment is far
        if (fw == -1 || id == skip || fw == skip) continue;
        float vx, vy, vz;
        if (R2 >= a.w && seg_vel32(f4, Rx, Ry, Rz, d.x, d.y, d.z, vx, vy, vz)) {
          bx += vx; by += vy; bz += vz;
        } else {
          const double* src = S.r1r2 + 6 * id;
          d3 v = seg_vel64(P.f4pi, mk3(src[0], src[1], src[2]), mk3(src[3], src[4], src[5]), r);
          ax += v.x; ay += v.y; az += v.z;
        }
      }
      ax += bx; ay += by; az += bz;
    }
  }
  if (k >= 0) {
    double* o = part + (size_t)j * 3 * stride + 3 * (size_t)k;
    o[0] = act ? ax : 0; o[1] = act ? ay : 0; o[2] = act ? az : 0;
  }
}

// v_nl = part[0]; v_img = sum_j part[j] in image order (src/tangle.c:627-638);
// mirror images reflect their velocity (src/tangle.c:633-634)
__global__ void k_reduce_images(OvParams P, const double* __restrict__ part, int n_t,
                                double* v_nl, double* v_img) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_t) return;
  d3 a = ld3(part, k);
  if (v_nl) st3(v_nl, k, a);
  d3 s = mk3(0, 0, 0);
  for (int j = 1; j <= P.n_img; ++j) {
    d3 v = ld3(part + (size_t)j * 3 * n_t, k);
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

bool ov_direct_nodes(ov_state_impl* s, const double* pos, double* v_nl, double* v_img) {
  if (s->n == 0) return true;
  if (!ensure_segtab(s, pos)) return false;
  int nimg = s->P.n_img;
  size_t bytes = sizeof(double) * 3 * (size_t)s->n * (nimg + 1);
  if (!s->img_part.reserve(bytes)) return false;
  dim3 grid((s->n + kTB - 1) / kTB, nimg + 1);
  SegTab S{s->seg64.as<double>(), s->segid.as<int>()};
  OvStatsAcc& st = ov_stats_tls();
  cudaEventRecord(s->ev1, s->stream);
  if (s->P.precision == OV_PREC_MIXED) {
    // spatially sorted order from the tree's key sort
    if (!ov_tree_build(s, pos, &s->tree)) return false;
    k_direct_mixed<<<dim3((s->tree.n_nodes + kTB - 1) / kTB, nimg + 1), kTB, 0, s->stream>>>(
        s->P, S, s->tree.n_nodes, pos, s->status.as<int2>(), s->tree.perm.as<int>(), s->tree.n_nodes,
        s->n, s->img_part.as<double>());
    OV_LAUNCHED();
    OV_TRY_CUDA(cudaGetLastError());
    // k_direct_mixed wrote part[j][k] for slots k in the sorted set only;
    // EMPTY slots are never read by the epilogue, but zero them for hygiene
  } else {
    k_direct64<<<grid, kTB, 0, s->stream>>>(s->P, S, s->n, nullptr, pos, s->status.as<int2>(),
                                            nullptr, s->n, s->img_part.as<double>());
    OV_LAUNCHED();
    OV_TRY_CUDA(cudaGetLastError());
  }
  cudaEventRecord(s->ev2, s->stream);
  k_reduce_images<<<(s->n + 255) / 256, 256, 0, s->stream>>>(s->P, s->img_part.as<double>(), s->n,
                                                              v_nl, v_img);
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
  size_t bytes = sizeof(double) * 3 * (size_t)npts * (nimg + 1);
  if (!s->img_part.reserve(bytes)) return false;
  dim3 grid((npts + kTB - 1) / kTB, nimg + 1);
  SegTab S{s->seg64.as<double>(), s->segid.as<int>()};
  int n_src = only ? n_only : s->n;
  k_direct64<<<grid, kTB, 0, s->stream>>>(s->P, S, n_src, only, pts, nullptr, skip, npts,
                                          s->img_part.as<double>());
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  // out_nl = part[0]; out_img = image sum in table order (src/tangle.c:624-638)
  OvParams P = s->P;
  P.n_img = nimg;
  k_reduce_images<<<(npts + 255) / 256, 256, 0, s->stream>>>(P, s->img_part.as<double>(), npts,
                                                              out_nl, out_img);
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
  k_direct64<<<grid, kTB, 0, st>>>(P, SegTab{seg, fwd}, n, nullptr, pts, nullptr, skip, npts, part);
  OV_LAUNCHED();
  k_reduce_images<<<(npts + 255) / 256, 256, 0, st>>>(P, part, npts, out, img);
  OV_LAUNCHED();
  k_add3<<<(3 * npts + 255) / 256, 256, 0, st>>>(out, img, out, npts);
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  return true;
}
