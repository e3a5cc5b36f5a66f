// ov_reconnect.cu - vortex-vortex reconnection with the candidate search on
// the GPU (ov_reconnect_candidates, ov_reconnect_vortices).
//
// The reference's pair loop (reconnect, src/vortex_dynamics.c:216-313)
// tests every pair k < l: both nodes neither empty nor pinned, not linked,
// distance after the periodic wrap (seg_pwrap) at most rec_dist, both
// tangents at least 0.5 long, tangents at an angle above rec_angle, nodes
// approaching each other; then do_reconnection swaps the links if that does
// not lengthen the tangle, and the nodes around a reconnection sit out the
// rest of the pass.  Positions and tangents do not change during a pass, so
// the distance, length and angle tests are the same before and after any
// reconnection of the pass: the GPU finds every pair passing them with a
// neighbour search on a hashed uniform grid (cells at least rec_dist wide,
// each node against the 27 cells around its own), in the reference's FP64
// operations.  The host then walks those pairs in the loop's order and
// applies what does change during the pass: the links, the sit-out flags,
// the approach test (update_velocity of both nodes, on the current links)
// and do_reconnection.
#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <vector>

#include "ov_internal.h"

namespace {

constexpr int kAxisBits = 21;
constexpr long long kAxisHalf = 1LL << (kAxisBits - 1);

struct Grid {
  double lo[3];
  double h[3];     // cell sizes (>= rec_dist)
  int G[3];        // cells per periodic axis (0: open axis, unbounded)
};

__device__ __forceinline__ long long cell_of(const Grid& g, int a, double x) {
  long long c = (long long)floor((x - g.lo[a]) / g.h[a]);
  if (g.G[a] > 0) {
    c %= g.G[a];
    if (c < 0) c += g.G[a];
  } else {
    c = max(-kAxisHalf, min(kAxisHalf - 1, c));
  }
  return c;
}

__device__ __forceinline__ unsigned long long key_of(long long cx, long long cy, long long cz) {
  return ((unsigned long long)(cx + kAxisHalf) << (2 * kAxisBits)) |
         ((unsigned long long)(cy + kAxisHalf) << kAxisBits) | (unsigned long long)(cz + kAxisHalf);
}

__device__ __forceinline__ bool eligible(int st) {
  return st != OV_EMPTY && st != OV_PINNED && st != OV_PINNED_SLIP;
}

__global__ void k_rec_keys(Grid g, const double* __restrict__ pos, const int2* __restrict__ status,
                           unsigned long long* keys, int* ids, int n) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  ids[m] = m;
  if (!eligible(status[m].x)) {
    keys[m] = ~0ULL;
    return;
  }
  const d3 p = ld3(pos, m);
  keys[m] = key_of(cell_of(g, 0, p.x), cell_of(g, 1, p.y), cell_of(g, 2, p.z));
}

// sqrt(((0 + x x) + y y) + z z): vec3_d (src/vec3_maths.c:338-345)
__device__ __forceinline__ double vec3_d_ref(d3 v) { return norm_ref(v); }

// dot(u, v) / |u| / |v| (vec3_ndot, src/vec3_maths.c:295-301)
__device__ __forceinline__ double ndot_ref(d3 u, d3 v) {
  double dot = __dmul_rn(u.x, v.x);
  dot = __dadd_rn(dot, __dmul_rn(u.y, v.y));
  dot = __dadd_rn(dot, __dmul_rn(u.z, v.z));
  return __ddiv_rn(__ddiv_rn(dot, vec3_d_ref(u)), vec3_d_ref(v));
}

// first index in keys[0, n) with keys[i] >= key
__device__ __forceinline__ int lower_bound(const unsigned long long* keys, int n, unsigned long long key) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (keys[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// One thread per node k: every l > k in the 27 cells around k's cell that
// passes the pass-invariant tests, appended to pairs (bounded by cap).
__global__ void k_rec_scan(OvParams P, Grid g, const double* __restrict__ pos, const int2* __restrict__ links,
                           const int2* __restrict__ status, const double* __restrict__ tan,
                           const unsigned long long* __restrict__ keys, const int* __restrict__ ids, int n,
                           double rec_dist, double cos_angle, int2* pairs, int cap, int* count) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n || !eligible(status[k].x)) return;
  const d3 pk = ld3(pos, k);
  const d3 tk = ld3(tan, k);
  if (vec3_d_ref(tk) < 0.5) return;
  const int2 lk = links[k];
  long long c[3] = {cell_of(g, 0, pk.x), cell_of(g, 1, pk.y), cell_of(g, 2, pk.z)};
  // distinct neighbour cells per axis
  long long nb[3][3];
  int nn[3];
  for (int a = 0; a < 3; ++a) {
    nn[a] = 0;
    for (int o = -1; o <= 1; ++o) {
      long long v = c[a] + o;
      if (g.G[a] > 0) {
        v %= g.G[a];
        if (v < 0) v += g.G[a];
      } else {
        v = max(-kAxisHalf, min(kAxisHalf - 1, v));
      }
      bool dup = false;
      for (int q = 0; q < nn[a]; ++q) dup |= nb[a][q] == v;
      if (!dup) nb[a][nn[a]++] = v;
    }
  }
  for (int ix = 0; ix < nn[0]; ++ix)
    for (int iy = 0; iy < nn[1]; ++iy)
      for (int iz = 0; iz < nn[2]; ++iz) {
        const unsigned long long key = key_of(nb[0][ix], nb[1][iy], nb[2][iz]);
        for (int i = lower_bound(keys, n, key); i < n && keys[i] == key; ++i) {
          const int l = ids[i];
          if (l <= k || lk.x == l || lk.y == l) continue;
          const d3 pl = pwrap(P, pk, ld3(pos, l));   // seg_pwrap: r1 = x_k, r2 = wrapped x_l
          if (vec3_d_ref(pk - pl) > rec_dist) continue;
          const d3 tl = ld3(tan, l);
          if (vec3_d_ref(tl) < 0.5) continue;
          if (ndot_ref(tk, tl) > cos_angle) continue;
          const int slot = atomicAdd(count, 1);
          if (slot < cap) pairs[slot] = make_int2(k, l);
        }
      }
}

// ---------------------------------------------------------------- velocities
// The approach test needs update_velocity (src/tangle.c:583-684) of both
// nodes on the links current at the test.  Velocities of the nodes of the
// next candidates come from one batched FP64 direct sum over all segments
// and images (ov_direct_points); after each reconnection every node computed
// so far gets the exact change: the two removed and the two added segments
// of do_reconnection over the tangle and all its images.  A node's epilogue
// (local term, flows, friction) then follows on the current links.

// targets of a batch: node positions, each skipping its own segments
// Every kernel below checks each listed slot against n (flag bit 1 and no
// access when outside), so a wrong list is an error, not a stray access.
__global__ void k_rec_points(const int* __restrict__ nodes, int count, int n, const double* __restrict__ pos,
                             double* pts, int* skip, int* flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int k = nodes[i];
  if (k < 0 || k >= n) {
    atomicOr(flag, 1);
    pts[3 * i] = pts[3 * i + 1] = pts[3 * i + 2] = 0;
    skip[i] = -1;
    return;
  }
  st3(pts, i, ld3(pos, k));
  skip[i] = k;
}

__global__ void k_rec_scatter(const int* __restrict__ nodes, int count, int n, const double* __restrict__ nl,
                              const double* __restrict__ img, double* v_nl, double* v_img, int* flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int k = nodes[i];
  if (k < 0 || k >= n) {
    atomicOr(flag, 1);
    return;
  }
  st3(v_nl, k, ld3(nl, i));
  st3(v_img, k, ld3(img, i));
}

// the four links do_reconnection changed, as kernel arguments
struct LinkPatch {
  int slot[4];
  int2 link[4];
};

__global__ void k_rec_patch_links(LinkPatch L, int2* links, int n, int* flag) {
  const int c = threadIdx.x;
  if (c >= 4) return;
  if (L.slot[c] < 0 || L.slot[c] >= n) {
    atomicOr(flag, 1);
    return;
  }
  links[L.slot[c]] = L.link[c];
}

// one segment change of a reconnection: slot m's forward link was (sign -1)
// or is now (sign +1) f
struct SegChange {
  int m[4], f[4];
  double sign[4];
};

// v_nl and v_img of the listed nodes += the changed segments' fields, with
// the skip rule of the tangle's own sum (src/tangle.c:614-616) and the
// mirror reflection of each image's sum (src/tangle.c:633-634).  One warp
// per node: lane 0 takes the tangle itself, the lanes share the images
// (image j on lane j mod 32), and the image terms are added in a fixed
// shuffle tree, so the result does not depend on scheduling.
constexpr int kCorrectWarps = 4;
__global__ void __launch_bounds__(32 * kCorrectWarps) k_rec_correct(OvParams P, SegChange C,
                                                                   const int* __restrict__ nodes, int count,
                                                                   int n, const double* __restrict__ pos,
                                                                   double* v_nl, double* v_img, int* flag) {
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * kCorrectWarps + (threadIdx.x >> 5);
  if (i >= count) return;   // whole warp
  const int k = nodes[i];
  bool ok = k >= 0 && k < n;
  for (int c = 0; c < 4; ++c) ok = ok && C.m[c] >= 0 && C.m[c] < n && C.f[c] >= 0 && C.f[c] < n;
  if (!ok) {
    if (lane == 0) atomicOr(flag, 1);
    return;
  }
  const d3 r = ld3(pos, k);
  d3 r1[4], r2[4];
  for (int c = 0; c < 4; ++c) {
    r1[c] = ld3(pos, C.m[c]);
    r2[c] = pwrap(P, r1[c], ld3(pos, C.f[c]));
  }
  d3 nl = mk3(0, 0, 0), im = mk3(0, 0, 0);
  if (lane == 0)
    for (int c = 0; c < 4; ++c)
      if (k != C.m[c] && k != C.f[c]) nl = nl + seg_vel64(P.f4pi, r1[c], r2[c], r) * C.sign[c];
  for (int j = lane; j < P.n_img; j += 32) {
    const d3 t = image_point(P, j, r);
    d3 v = mk3(0, 0, 0);
    for (int c = 0; c < 4; ++c) v = v + seg_vel64(P.f4pi, r1[c], r2[c], t) * C.sign[c];
    const int face = P.img[j][3];
    if (face > -1) v = mirror_dir(v, face);
    im = im + v;
  }
  for (int off = 16; off > 0; off >>= 1) {
    im.x += __shfl_down_sync(0xffffffffu, im.x, off);
    im.y += __shfl_down_sync(0xffffffffu, im.y, off);
    im.z += __shfl_down_sync(0xffffffffu, im.z, off);
  }
  if (lane == 0) {
    st3(v_nl, k, ld3(v_nl, k) + nl);
    st3(v_img, k, ld3(v_img, k) + im);
  }
}

// vels and vs of the listed nodes, packed 6 doubles per node for one copy
__global__ void k_rec_pack(const int* __restrict__ nodes, int count, int n, const double* __restrict__ vels,
                           const double* __restrict__ vs, double* out, int* flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int k = nodes[i];
  if (k < 0 || k >= n) {
    atomicOr(flag, 1);
    for (int c = 0; c < 6; ++c) out[6 * (size_t)i + c] = 0;
    return;
  }
  st3(out + 6 * (size_t)i, 0, ld3(vels, k));
  st3(out + 6 * (size_t)i + 3, 0, ld3(vs, k));
}

// Pinned host memory for the pass's per-reconnection copies (the known list
// up, the known nodes' values and the error flag down), so each copy is one
// asynchronous transfer rather than a staged pageable one.
struct PinnedBuf {
  void* p = nullptr;
  size_t bytes = 0;
  bool reserve(size_t n) {
    if (n <= bytes) return true;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    if (!ov_cuda_ok(cudaMallocHost(&p, n), "cudaMallocHost")) return false;
    bytes = n;
    return true;
  }
  template <class T> T* as() const { return static_cast<T*>(p); }
  ~PinnedBuf() {
    if (p) cudaFreeHost(p);
  }
};

struct RecState {
  PinnedBuf h_list, h_vals;   // known list (ints), known values (6 doubles each) + flag
  ov_state_impl s;
  DevBuf keys, keys2, ids, ids2, pairs, count, hist, scan_part, skip, pack;
  DevBuf batch, pts, bnl, bimg, known;   // batched velocities
  DevBuf bound, two;                     // mixed form: error bounds, FP64 re-checks
};

// counters of the last ov_reconnect_vortices call on this thread
thread_local ov_reconnect_stats g_rec_stats;

double secs_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

RecState& rec_state() {
  static thread_local RecState r;
  return r;
}

// host restatements of the reference's vector helpers (src/vec3_maths.c)
double h_d(const double* v) {
  double out = 0;
  for (int c = 0; c < 3; ++c) out += v[c] * v[c];
  return sqrt(out);
}

void h_pwrap(const tangle_state* t, const double* r1, const double* r2, double* out) {
  for (int c = 0; c < 3; ++c) {
    out[c] = r2[c];
    if (t->box.wall[2 * c] != WALL_PERIODIC) continue;
    const double L = t->box.top_right_front.p[c] - t->box.bottom_left_back.p[c];
    const double d = r2[c] - r1[c];
    if (d > L / 2) out[c] -= L;
    else if (d < -L / 2) out[c] += L;
  }
}

double h_seglen(const tangle_state* t, int a, int b) {
  double w[3], d[3];
  h_pwrap(t, t->vnodes[a].p, t->vnodes[b].p, w);
  for (int c = 0; c < 3; ++c) d[c] = w[c] - t->vnodes[a].p[c];
  return h_d(d);
}

// do_reconnection (src/vortex_dynamics.c:317-364): swap the links of k and
// l unless both ways lengthen the tangle; the changed slots are returned
bool do_reconnection(tangle_state* t, int k, int l, int changed[4]) {
  const int kf = t->connections[k].forward, kr = t->connections[k].reverse;
  const int lf = t->connections[l].forward, lr = t->connections[l].reverse;
  const double kl = h_seglen(t, k, l);
  const double cf1 = kl + h_seglen(t, kf, lr) - h_seglen(t, k, kf) - h_seglen(t, l, lr);
  const double cf2 = kl + h_seglen(t, kr, lf) - h_seglen(t, k, kr) - h_seglen(t, l, lf);
  if (cf1 > 0 && cf2 > 0) return false;
  if (cf1 < cf2) {
    t->connections[k].forward = l;
    t->connections[l].reverse = k;
    t->connections[kf].reverse = lr;
    t->connections[lr].forward = kf;
    changed[0] = k; changed[1] = l; changed[2] = kf; changed[3] = lr;
  } else {
    t->connections[l].forward = k;
    t->connections[k].reverse = l;
    t->connections[lf].reverse = kr;
    t->connections[kr].forward = lf;
    changed[0] = l; changed[1] = k; changed[2] = lf; changed[3] = kr;
  }
  return true;
}

bool find_candidates(RecState& R, const tangle_state* t, double rec_dist, double rec_angle,
                     std::vector<int2>& out) {
  ov_state_impl* s = &R.s;
  const int n = t->N;
  out.clear();
  if (n == 0) return true;
  Grid g;
  for (int a = 0; a < 3; ++a) {
    g.lo[a] = s->P.lo[a];
    if (s->P.periodic[a]) {
      const double L = s->P.L[a];
      int G = (int)std::min(1e6, std::max(1.0, floor(L / rec_dist)));
      g.G[a] = G;
      g.h[a] = L / G;
    } else {
      g.G[a] = 0;
      g.h[a] = rec_dist;
    }
  }
  const size_t nk = (size_t)n;
  if (!R.keys.reserve(8 * nk) || !R.keys2.reserve(8 * nk) || !R.ids.reserve(4 * nk) ||
      !R.ids2.reserve(4 * nk) || !R.count.reserve(64))
    return false;
  k_rec_keys<<<(n + 255) / 256, 256, 0, s->stream>>>(g, s->pos.as<double>(), s->status.as<int2>(),
                                                     R.keys.as<unsigned long long>(), R.ids.as<int>(), n);
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  // the tree build's radix sort; the sorted keys and ids end in keys / ids
  if (!ov_radix_sort_u64(R.keys.as<uint64_t>(), R.ids.as<int>(), R.keys2.as<uint64_t>(), R.ids2.as<int>(), n,
                         R.hist, R.scan_part, s->stream))
    return false;
  int cap = std::max(1024, n / 4);
  const double cos_angle = cos(rec_angle);
  for (int attempt = 0; attempt < 2; ++attempt) {
    if (!R.pairs.reserve(sizeof(int2) * (size_t)cap)) return false;
    OV_TRY_CUDA(cudaMemsetAsync(R.count.p, 0, sizeof(int), s->stream));
    k_rec_scan<<<(n + 127) / 128, 128, 0, s->stream>>>(
        s->P, g, s->pos.as<double>(), s->links.as<int2>(), s->status.as<int2>(), s->tan.as<double>(),
        R.keys.as<unsigned long long>(), R.ids.as<int>(), n, rec_dist, cos_angle, R.pairs.as<int2>(), cap,
        R.count.as<int>());
    OV_LAUNCHED();
    OV_TRY_CUDA(cudaGetLastError());
    int cnt = 0;
    OV_TRY_CUDA(cudaMemcpyAsync(&cnt, R.count.p, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    OV_TRY_CUDA(cudaStreamSynchronize(s->stream));
    if (cnt <= cap) {
      out.resize(cnt);
      if (cnt)
        OV_TRY_CUDA(cudaMemcpy(out.data(), R.pairs.p, sizeof(int2) * (size_t)cnt, cudaMemcpyDeviceToHost));
      // the reference's loop order: k ascending, then l ascending
      std::sort(out.begin(), out.end(), [](const int2& a, const int2& b) {
        return a.x != b.x ? a.x < b.x : a.y < b.y;
      });
      return true;
    }
    cap = cnt;   // exact size for the second scan
  }
  ov_set_error(OV_ERR_CUDA, "reconnection candidate count changed between two scans");
  return false;
}

bool upload_for_pass(RecState& R, const tangle_state* t) {
  ov_state_impl* s = &R.s;
  if (!ov_upload_tangle(s, t)) return false;
  if (t->N > 0 && (!t->tangents || !t->normals)) {
    ov_set_error(OV_ERR_INVALID, "reconnection needs the tangle's tangents and normals");
    return false;
  }
  const size_t v3 = 24 * (size_t)t->N;
  if (t->N > 0) {
    OV_TRY_CUDA(cudaMemcpyAsync(s->tan.p, t->tangents, v3, cudaMemcpyHostToDevice, s->stream));
    OV_TRY_CUDA(cudaMemcpyAsync(s->nrm.p, t->normals, v3, cudaMemcpyHostToDevice, s->stream));
  }
  return true;
}

// Velocities (vels, vs) of the nodes known so far, as the device holds them
// on the current links, mirrored on the host: node k's values at
// hv[6 * pos_of[k]].
struct RecVel {
  std::vector<int> known;        // slots with velocities on the device
  std::vector<int> pos_of;       // slot -> index in known, -1 if not known
  std::vector<double> hv;        // 6 per known node: vels, vs
  std::vector<double> bound;     // per known node: bound on |mixed - FP64| of its sums (0: FP64)
  double time = 0;
};

// epilogue of every known node and the copy of their vels and vs to the host
bool refresh_known(RecState& R, RecVel& V) {
  ov_state_impl* s = &R.s;
  const int cnt = (int)V.known.size();
  if (cnt == 0) return true;
  // the pass's error flag (zeroed at its start) accumulates every kernel's bits
  int* flag = s->dflag.as<int>();
  if (!ov_launch_epilogue_list(s->stream, s->P, s->links.as<int2>(), s->status.as<int2>(), V.time,
                               s->pos.as<double>(), s->tan.as<double>(), s->nrm.as<double>(),
                               s->v_nl.as<double>(), s->v_img.as<double>(), s->vels.as<double>(),
                               s->vs.as<double>(), R.known.as<int>(), cnt, flag))
    return false;
  if (!R.pack.reserve(sizeof(double) * 6 * (size_t)cnt + 64)) return false;
  k_rec_pack<<<(cnt + 255) / 256, 256, 0, s->stream>>>(R.known.as<int>(), cnt, s->n, s->vels.as<double>(),
                                                       s->vs.as<double>(), R.pack.as<double>(), flag);
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  // the values, then the flag, into pinned memory: one wait
  const size_t vbytes = sizeof(double) * 6 * (size_t)cnt;
  if (!R.h_vals.reserve(vbytes + 64)) return false;
  int* h_flag = reinterpret_cast<int*>(R.h_vals.as<char>() + vbytes);
  OV_TRY_CUDA(cudaMemcpyAsync(R.h_vals.p, R.pack.p, vbytes, cudaMemcpyDeviceToHost, s->stream));
  OV_TRY_CUDA(cudaMemcpyAsync(h_flag, flag, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  OV_TRY_CUDA(cudaStreamSynchronize(s->stream));
  V.hv.assign(R.h_vals.as<double>(), R.h_vals.as<double>() + 6 * (size_t)cnt);
  return ov_flag_status(*h_flag, "update_velocity");
}

// the known list to the device (R.known), through pinned memory.  Every
// upload is followed by refresh_known's wait before the next one, so the
// pinned list is never rewritten while a copy from it is in flight.
bool upload_known(RecState& R, const RecVel& V) {
  const size_t cnt = V.known.size();
  if (cnt == 0) return true;
  if (!R.known.reserve(sizeof(int) * cnt) || !R.h_list.reserve(sizeof(int) * cnt)) return false;
  std::copy(V.known.begin(), V.known.end(), R.h_list.as<int>());
  OV_TRY_CUDA(cudaMemcpyAsync(R.known.p, R.h_list.p, sizeof(int) * cnt, cudaMemcpyHostToDevice, R.s.stream));
  return true;
}

// Nonlocal and image sums of the m nodes at `batch` (a device list) on the
// current links into v_nl, v_img: FP64, or (mixed) the FP32 far field with
// a bound on its error per node copied into hb.
bool sum_nodes(RecState& R, const int* batch, int m, bool mixed, double* hb) {
  ov_state_impl* s = &R.s;
  if (!R.pts.reserve(sizeof(double) * 3 * (size_t)m) || !R.skip.reserve(sizeof(int) * (size_t)m) ||
      !R.bnl.reserve(sizeof(double) * 3 * (size_t)m) || !R.bimg.reserve(sizeof(double) * 3 * (size_t)m) ||
      !R.bound.reserve(sizeof(double) * (size_t)m))
    return false;
  k_rec_points<<<(m + 255) / 256, 256, 0, s->stream>>>(batch, m, s->n, s->pos.as<double>(), R.pts.as<double>(),
                                                        R.skip.as<int>(), s->dflag.as<int>());
  OV_LAUNCHED();
  const bool ok = mixed ? ov_direct_points_bounded(s, s->pos.as<double>(), m, R.pts.as<double>(),
                                                   R.skip.as<int>(), R.bnl.as<double>(), R.bimg.as<double>(),
                                                   R.bound.as<double>())
                        : ov_direct_points(s, s->pos.as<double>(), m, R.pts.as<double>(), R.skip.as<int>(),
                                           nullptr, 0, R.bnl.as<double>(), R.bimg.as<double>());
  if (!ok) return false;
  k_rec_scatter<<<(m + 255) / 256, 256, 0, s->stream>>>(batch, m, s->n, R.bnl.as<double>(), R.bimg.as<double>(),
                                                         s->v_nl.as<double>(), s->v_img.as<double>(),
                                                         s->dflag.as<int>());
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  if (mixed)
    OV_TRY_CUDA(cudaMemcpyAsync(hb, R.bound.p, sizeof(double) * (size_t)m, cudaMemcpyDeviceToHost, s->stream));
  return true;
}

// Sums of new nodes on the current links (one batched direct sum), added to
// the known set; then every known node's epilogue and host copy.
bool compute_nodes(RecState& R, RecVel& V, const std::vector<int>& nodes, bool mixed) {
  ov_state_impl* s = &R.s;
  const int m = (int)nodes.size();
  if (m == 0) return true;
  const int old = (int)V.known.size();
  for (int k : nodes) {
    V.pos_of[k] = (int)V.known.size();
    V.known.push_back(k);
  }
  const int cnt = (int)V.known.size();
  V.bound.resize(cnt, 0.0);
  // the whole list: growing R.known reallocates it without its contents
  if (!upload_known(R, V)) return false;
  const auto t0 = std::chrono::steady_clock::now();
  if (!s->P.lia_only && !sum_nodes(R, R.known.as<int>() + old, m, mixed, V.bound.data() + old)) return false;
  OV_TRY_CUDA(cudaStreamSynchronize(s->stream));
  g_rec_stats.sums_s += secs_since(t0);
  g_rec_stats.nodes_summed += m;
  return refresh_known(R, V);
}

// Both nodes of a candidate again with FP64 sums on the current links (the
// mixed sums left the approach test's sign open); the known set's other
// nodes keep their values.
bool recheck_fp64(RecState& R, RecVel& V, int k, int l) {
  ov_state_impl* s = &R.s;
  const int two[2] = {k, l};
  if (!R.two.reserve(sizeof(int) * 2)) return false;
  const auto t0 = std::chrono::steady_clock::now();
  OV_TRY_CUDA(cudaMemcpyAsync(R.two.p, two, sizeof(two), cudaMemcpyHostToDevice, s->stream));
  if (!s->P.lia_only && !sum_nodes(R, R.two.as<int>(), 2, false, nullptr)) return false;
  OV_TRY_CUDA(cudaStreamSynchronize(s->stream));
  g_rec_stats.sums_s += secs_since(t0);
  V.bound[V.pos_of[k]] = 0.0;
  V.bound[V.pos_of[l]] = 0.0;
  ++g_rec_stats.fp64_rechecks;
  return refresh_known(R, V);
}

}  // namespace

extern "C" {

int ov_reconnect_candidates(const struct tangle_state* tangle, double rec_dist, double rec_angle, int* pairs,
                            int max_pairs) {
  ov_clear_error();
  if (!tangle || rec_dist <= 0 || max_pairs < 0 || (max_pairs > 0 && !pairs)) {
    ov_set_error(OV_ERR_INVALID, "ov_reconnect_candidates: null tangle/output or rec_dist <= 0");
    return -OV_ERR_INVALID;
  }
  RecState& R = rec_state();
  std::vector<int2> c;
  if (!upload_for_pass(R, tangle) || !find_candidates(R, tangle, rec_dist, rec_angle, c)) return -ov_last_error();
  const int m = std::min<int>((int)c.size(), max_pairs);
  for (int i = 0; i < m; ++i) {
    pairs[2 * i] = c[i].x;
    pairs[2 * i + 1] = c[i].y;
  }
  return (int)c.size();
}

int ov_reconnect_vortices(struct tangle_state* tangle, double t, double rec_dist, double rec_angle) {
  ov_clear_error();
  if (!tangle || rec_dist <= 0 || (tangle->N > 0 && (!tangle->recalculate || !tangle->vels || !tangle->vs))) {
    ov_set_error(OV_ERR_INVALID, "ov_reconnect_vortices: null tangle, arrays or rec_dist <= 0");
    return -OV_ERR_INVALID;
  }
  RecState& R = rec_state();
  std::vector<int2> cand;
  const auto t_start = std::chrono::steady_clock::now();
  g_rec_stats = ov_reconnect_stats{};
  if (!upload_for_pass(R, tangle) || !find_candidates(R, tangle, rec_dist, rec_angle, cand))
    return -ov_last_error();
  g_rec_stats.search_s = secs_since(t_start);
  ov_state_impl* s = &R.s;
  if (!ov_cuda_ok(cudaMemsetAsync(s->dflag.p, 0, sizeof(int), s->stream), "cudaMemsetAsync"))
    return -ov_last_error();
  RecVel V;
  V.pos_of.assign(tangle->N, -1);
  V.time = t;
  g_rec_stats.candidates = (int)cand.size();
  // Mixed form: the approach test's sums with the FP32 far field and a
  // bound E on their error per node.  vels is affine in the sums (the
  // epilogue, src/tangle.c:643-684, adds terms of the local velocity and of
  // t' x (v_n - v_s) and t' x (t' x (v_n - v_s))), so vels moves by at most
  // (1 + |alpha| |t'| + |alpha'| |t'|^2) E, and dx . dv by |dx| times the
  // two nodes' sum of that.  A test whose |dx . dv| is within it (plus
  // 1e-13 of |dx| (|v_k| + |v_l|) for the FP64 arithmetic) is taken again
  // with FP64 sums, so every decision is the FP64 form's.
  const bool mixed = s->P.precision == OV_PREC_MIXED;
  // OV_RECONNECT_MARGIN_SCALE multiplies that margin (a huge value takes
  // every mixed test again in FP64; for tests of this path)
  double margin_scale = 1.0;
  if (const char* e = getenv("OV_RECONNECT_MARGIN_SCALE")) margin_scale = atof(e);
  auto amp = [&](int k) {
    if (!s->P.use_mf) return 1.0;
    const double* tk = tangle->tangents[k].p;
    const double tn = sqrt(tk[0] * tk[0] + tk[1] * tk[1] + tk[2] * tk[2]);
    return 1.0 + fabs(s->P.alpha) * tn + fabs(s->P.alpha_p) * tn * tn;
  };
  // the nodes of this many upcoming candidates per batched direct sum
  constexpr int kBatchNodes = 2048;
  // recalculate holds the sit-out flags on entry: the reference zeroes them
  // at the top of reconnect (src/vortex_dynamics.c:148-149), before its wall
  // part, whose reconnections the loop then leaves alone
  auto linked = [&](int k, int l) {
    return tangle->connections[k].forward == l || tangle->connections[k].reverse == l;
  };
  int nrecs = 0, done_k = -1;
  for (size_t i = 0; i < cand.size(); ++i) {
    const int k = cand[i].x, l = cand[i].y;
    // after a reconnection the reference leaves k's inner loop
    if (k == done_k || tangle->recalculate[k] || tangle->recalculate[l] || linked(k, l)) continue;
    if (V.pos_of[k] == -1 || V.pos_of[l] == -1) {
      // velocities of the nodes of the next candidates that can still be
      // tested (some may be skipped after later reconnections)
      std::vector<int> batch;
      for (size_t j = i; j < cand.size() && (int)batch.size() < kBatchNodes; ++j) {
        const int a = cand[j].x, b = cand[j].y;
        if (tangle->recalculate[a] || tangle->recalculate[b] || linked(a, b)) continue;
        for (int x : {a, b})
          if (V.pos_of[x] == -1) {
            V.pos_of[x] = -2;   // queued
            batch.push_back(x);
          }
      }
      for (int x : batch) V.pos_of[x] = -1;
      if (!compute_nodes(R, V, batch, mixed)) return -ov_last_error();
    }
    ++g_rec_stats.tested;
    // approach test (src/vortex_dynamics.c:266-281) on the known values
    double w[3], dx[3];
    h_pwrap(tangle, tangle->vnodes[k].p, tangle->vnodes[l].p, w);
    for (int c = 0; c < 3; ++c) dx[c] = tangle->vnodes[k].p[c] - w[c];
    auto approach = [&](double& dot, double& scale) {
      const double* hk = V.hv.data() + 6 * (size_t)V.pos_of[k];
      const double* hl = V.hv.data() + 6 * (size_t)V.pos_of[l];
      dot = 0;
      double vk2 = 0, vl2 = 0;
      for (int c = 0; c < 3; ++c) {
        dot += dx[c] * (hk[c] - hl[c]);
        vk2 += hk[c] * hk[c];
        vl2 += hl[c] * hl[c];
      }
      scale = sqrt(vk2) + sqrt(vl2);
    };
    double dot, vscale;
    approach(dot, vscale);
    if (mixed) {
      const double ek = V.bound[V.pos_of[k]], el = V.bound[V.pos_of[l]];
      const double dxn = sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
      const double margin = margin_scale * dxn * (amp(k) * ek + amp(l) * el + 1e-13 * vscale);
      if ((ek > 0 || el > 0) && !(fabs(dot) > margin)) {
        if (!recheck_fp64(R, V, k, l)) return -ov_last_error();
        approach(dot, vscale);
      }
    }
    // update_velocity of both nodes writes their vels and vs (as the
    // reference's does, src/vortex_dynamics.c:275-276)
    {
      const double* hk = V.hv.data() + 6 * (size_t)V.pos_of[k];
      const double* hl = V.hv.data() + 6 * (size_t)V.pos_of[l];
      for (int c = 0; c < 3; ++c) {
        tangle->vels[k].p[c] = hk[c];
        tangle->vs[k].p[c] = hk[3 + c];
        tangle->vels[l].p[c] = hl[c];
        tangle->vs[l].p[c] = hl[3 + c];
      }
    }
    if (dot > 0) continue;
    const int knext = tangle->connections[k].forward, kprev = tangle->connections[k].reverse;
    const int lnext = tangle->connections[l].forward, lprev = tangle->connections[l].reverse;
    int changed[4], old_fwd[2];
    if (!do_reconnection(tangle, k, l, changed)) continue;
    // changed[0] and changed[3] are the slots whose forward link changed:
    // k (was kf) and lr (was l), or l (was lf) and kr (was k)
    old_fwd[0] = changed[0] == k ? knext : lnext;
    old_fwd[1] = changed[0] == k ? l : k;
    // the same links on the device
    {
      LinkPatch L;
      for (int c = 0; c < 4; ++c) {
        L.slot[c] = changed[c];
        L.link[c] = make_int2(tangle->connections[changed[c]].forward, tangle->connections[changed[c]].reverse);
      }
      k_rec_patch_links<<<1, 32, 0, s->stream>>>(L, s->links.as<int2>(), s->n, s->dflag.as<int>());
      OV_LAUNCHED();
      if (!ov_cuda_ok(cudaGetLastError(), "k_rec_patch_links")) return -ov_last_error();
    }
    const int flag[10] = {k, tangle->connections[k].forward, tangle->connections[k].reverse, knext, kprev,
                          l, tangle->connections[l].forward, tangle->connections[l].reverse, lnext, lprev};
    for (int f : flag) tangle->recalculate[f]++;
    ++nrecs;
    done_k = k;
    // nodes now flagged sit out the rest of the pass: no more velocities for
    // them (a node whose own links changed may even sit on a zero-length
    // segment, whose local term is not finite)
    {
      std::vector<int> keep;
      std::vector<double> keep_bound;
      keep.reserve(V.known.size());
      keep_bound.reserve(V.known.size());
      for (size_t q = 0; q < V.known.size(); ++q) {
        const int x = V.known[q];
        if (tangle->recalculate[x]) {
          V.pos_of[x] = -3;   // retired
        } else {
          V.pos_of[x] = (int)keep.size();
          keep.push_back(x);
          keep_bound.push_back(V.bound[q]);
        }
      }
      V.known.swap(keep);
      V.bound.swap(keep_bound);
      if (!upload_known(R, V)) return -ov_last_error();
    }
    // every known node: the removed and added segments' fields
    SegChange C;
    C.m[0] = changed[0]; C.f[0] = old_fwd[0]; C.sign[0] = -1;
    C.m[1] = changed[3]; C.f[1] = old_fwd[1]; C.sign[1] = -1;
    C.m[2] = changed[0]; C.f[2] = tangle->connections[changed[0]].forward; C.sign[2] = 1;
    C.m[3] = changed[3]; C.f[3] = tangle->connections[changed[3]].forward; C.sign[3] = 1;
    const int cnt = (int)V.known.size();
    if (cnt > 0 && !s->P.lia_only) {
      k_rec_correct<<<(cnt + kCorrectWarps - 1) / kCorrectWarps, 32 * kCorrectWarps, 0, s->stream>>>(
          s->P, C, R.known.as<int>(), cnt, s->n, s->pos.as<double>(), s->v_nl.as<double>(),
          s->v_img.as<double>(), s->dflag.as<int>());
      OV_LAUNCHED();
      if (!ov_cuda_ok(cudaGetLastError(), "k_rec_correct")) return -ov_last_error();
    }
    if (!refresh_known(R, V)) return -ov_last_error();
  }
  if (!ov_cuda_ok(cudaStreamSynchronize(s->stream), "cudaStreamSynchronize")) return -ov_last_error();
  g_rec_stats.reconnections = nrecs;
  g_rec_stats.total_s = secs_since(t_start);
  return nrecs;
}

int ov_reconnect_get_stats(ov_reconnect_stats* out) {
  if (!out) {
    ov_set_error(OV_ERR_INVALID, "ov_reconnect_get_stats: null output");
    return -OV_ERR_INVALID;
  }
  *out = g_rec_stats;
  return 0;
}

}  // extern "C"
