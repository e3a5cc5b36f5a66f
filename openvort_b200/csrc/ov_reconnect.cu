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
#include <cub/device/device_radix_sort.cuh>
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
// The nonlocal and image sums (update_velocity's loops, src/tangle.c:611-636)
// at the two nodes of a candidate pair, spread over the whole GPU: block
// (c, j) sums segments [c chunk, (c + 1) chunk) at image j of both nodes,
// reduced in a fixed order in shared memory; k_pair_reduce then adds the
// blocks in order.
constexpr int kPV = 256;

struct SegRef {
  const double* r1r2;   // 6 doubles per slot: r1, wrapped r2 (k_segtab)
  const int* fwd;
};

__global__ void __launch_bounds__(kPV) k_pair_vel(OvParams P, SegRef S, int n, const double* __restrict__ pos,
                                                  int2 tk, int chunk, double* __restrict__ partial) {
  __shared__ double red[kPV][6];
  const int c = blockIdx.x, j = blockIdx.y, nch = gridDim.x;
  d3 r[2];
  int skip[2];
  const int t2[2] = {tk.x, tk.y};
#pragma unroll
  for (int u = 0; u < 2; ++u) {
    r[u] = ld3(pos, t2[u]);
    skip[u] = -1;
    if (j > 0) r[u] = image_point(P, j - 1, r[u]);
    else skip[u] = t2[u];
  }
  double a[6] = {0, 0, 0, 0, 0, 0};
  const int hi = min(n, (c + 1) * chunk);
  for (int m = c * chunk + threadIdx.x; m < hi; m += kPV) {
    const int fw = S.fwd[m];
    if (fw < 0) continue;
    const double* sg = S.r1r2 + 6 * (size_t)m;
    const d3 r1 = mk3(sg[0], sg[1], sg[2]), r2 = mk3(sg[3], sg[4], sg[5]);
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      if (m == skip[u] || fw == skip[u]) continue;
      const d3 v = seg_vel64(P.f4pi, r1, r2, r[u]);
      a[3 * u] += v.x;
      a[3 * u + 1] += v.y;
      a[3 * u + 2] += v.z;
    }
  }
#pragma unroll
  for (int q = 0; q < 6; ++q) red[threadIdx.x][q] = a[q];
  __syncthreads();
  for (int s = kPV / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int q = 0; q < 6; ++q) red[threadIdx.x][q] += red[threadIdx.x + s][q];
    __syncthreads();
  }
  if (threadIdx.x < 6) partial[((size_t)j * nch + c) * 6 + threadIdx.x] = red[0][threadIdx.x];
}

// v_nl and v_img of both nodes from the blocks' partial sums, in order;
// mirror images reflect their velocity (src/tangle.c:633-634)
__global__ void k_pair_reduce(OvParams P, const double* __restrict__ partial, int nch, int2 tk,
                              double* v_nl, double* v_img) {
  const int u = threadIdx.x;
  if (u >= 2) return;
  d3 nl = mk3(0, 0, 0), im = mk3(0, 0, 0);
  for (int c = 0; c < nch; ++c) nl = nl + ld3(partial + (size_t)c * 6, u);
  for (int j = 1; j <= P.n_img; ++j) {
    d3 v = mk3(0, 0, 0);
    for (int c = 0; c < nch; ++c) v = v + ld3(partial + ((size_t)j * nch + c) * 6, u);
    const int face = P.img[j - 1][3];
    if (face > -1) v = mirror_dir(v, face);
    im = im + v;
  }
  const int k = u == 0 ? tk.x : tk.y;
  st3(v_nl, k, nl);
  st3(v_img, k, im);
}

// vels and vs of nodes k and l and the status flag, packed for one copy
__global__ void k_pair_pack(const double* __restrict__ vels, const double* __restrict__ vs, int2 tk,
                            const int* __restrict__ flag, double* out) {
  const int i = threadIdx.x;
  if (i < 12) {
    const int node = i < 6 ? tk.x : tk.y, c = i % 3;
    out[i] = (i % 6 < 3 ? vels : vs)[3 * (size_t)node + c];
  }
  if (i == 12) out[12] = (double)*flag;
}

struct RecState {
  ov_state_impl s;
  DevBuf keys, keys2, ids, ids2, pairs, count, tmp, skip, partial, pack;
};

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
  size_t tmp_bytes = 0;
  OV_TRY_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, R.keys.as<unsigned long long>(),
                                              R.keys2.as<unsigned long long>(), R.ids.as<int>(),
                                              R.ids2.as<int>(), n, 0, 64, s->stream));
  if (!R.tmp.reserve(std::max<size_t>(tmp_bytes, 16))) return false;
  OV_TRY_CUDA(cub::DeviceRadixSort::SortPairs(R.tmp.p, tmp_bytes, R.keys.as<unsigned long long>(),
                                              R.keys2.as<unsigned long long>(), R.ids.as<int>(),
                                              R.ids2.as<int>(), n, 0, 64, s->stream));
  int cap = std::max(1024, n / 4);
  const double cos_angle = cos(rec_angle);
  for (int attempt = 0; attempt < 2; ++attempt) {
    if (!R.pairs.reserve(sizeof(int2) * (size_t)cap)) return false;
    OV_TRY_CUDA(cudaMemsetAsync(R.count.p, 0, sizeof(int), s->stream));
    k_rec_scan<<<(n + 127) / 128, 128, 0, s->stream>>>(
        s->P, g, s->pos.as<double>(), s->links.as<int2>(), s->status.as<int2>(), s->tan.as<double>(),
        R.keys2.as<unsigned long long>(), R.ids2.as<int>(), n, rec_dist, cos_angle, R.pairs.as<int2>(), cap,
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

// update_velocity (src/tangle.c:583-684) of nodes k and l on the resident
// state (direct sum: the reference passes no tree here), written back to
// the tangle's vels and vs
bool pair_velocity(RecState& R, tangle_state* t, int k, int l, double time) {
  ov_state_impl* s = &R.s;
  const int n = s->n;
  const int2 tk = make_int2(k, l);
  if (!s->P.lia_only) {
    // segment table of the current links
    if (!ov_segment_table(s, s->pos.as<double>())) return false;
    const int nimg = s->P.n_img;
    static int sms = 0;
    if (!sms) {
      int dev = 0;
      cudaGetDevice(&dev);
      if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 1;
    }
    // about 8 blocks of 256 threads per SM: the FP64 sum is latency-bound
    const int want = std::max(1, (8 * sms + nimg) / (nimg + 1));
    const int chunk = std::max(kPV, (n + want - 1) / want);
    const int nch = (n + chunk - 1) / chunk;
    if (!R.partial.reserve(sizeof(double) * 6 * (size_t)nch * (nimg + 1))) return false;
    k_pair_vel<<<dim3(nch, nimg + 1), kPV, 0, s->stream>>>(s->P, SegRef{s->seg64.as<double>(), s->segid.as<int>()},
                                                           n, s->pos.as<double>(), tk, chunk, R.partial.as<double>());
    OV_LAUNCHED();
    k_pair_reduce<<<1, 32, 0, s->stream>>>(s->P, R.partial.as<double>(), nch, tk, s->v_nl.as<double>(),
                                           s->v_img.as<double>());
    OV_LAUNCHED();
    OV_TRY_CUDA(cudaGetLastError());
  }
  int* flag = s->dflag.as<int>();
  OV_TRY_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s->stream));
  for (int u = 0; u < 2; ++u) {
    const int m = u == 0 ? k : l;
    if (!ov_launch_epilogue(s->stream, s->P, s->links.as<int2>(), s->status.as<int2>(), nullptr, time,
                            s->pos.as<double>(), s->tan.as<double>(), s->nrm.as<double>(), s->v_nl.as<double>(),
                            s->v_img.as<double>(), s->vels.as<double>(), s->vs.as<double>(), m, m + 1, flag))
      return false;
  }
  if (!R.pack.reserve(sizeof(double) * 13)) return false;
  k_pair_pack<<<1, 32, 0, s->stream>>>(s->vels.as<double>(), s->vs.as<double>(), tk, flag, R.pack.as<double>());
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  double h[13];
  OV_TRY_CUDA(cudaMemcpyAsync(h, R.pack.p, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
  OV_TRY_CUDA(cudaStreamSynchronize(s->stream));
  for (int c = 0; c < 3; ++c) {
    t->vels[k].p[c] = h[c];
    t->vs[k].p[c] = h[3 + c];
    t->vels[l].p[c] = h[6 + c];
    t->vs[l].p[c] = h[9 + c];
  }
  return ov_flag_status((int)h[12], "update_velocity");
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
  if (!upload_for_pass(R, tangle) || !find_candidates(R, tangle, rec_dist, rec_angle, cand))
    return -ov_last_error();
  // recalculate holds the sit-out flags on entry: the reference zeroes them
  // at the top of reconnect (src/vortex_dynamics.c:148-149), before its wall
  // part, whose reconnections the loop then leaves alone
  int nrecs = 0, done_k = -1;
  for (const int2& pr : cand) {
    const int k = pr.x, l = pr.y;
    // after a reconnection the reference leaves k's inner loop
    if (k == done_k || tangle->recalculate[k] || tangle->recalculate[l]) continue;
    if (tangle->connections[k].forward == l || tangle->connections[k].reverse == l) continue;
    // approach test on the current links (src/vortex_dynamics.c:266-277)
    if (!pair_velocity(R, tangle, k, l, t)) return -ov_last_error();
    double w[3], dx[3], dv[3];
    h_pwrap(tangle, tangle->vnodes[k].p, tangle->vnodes[l].p, w);
    for (int c = 0; c < 3; ++c) {
      dx[c] = tangle->vnodes[k].p[c] - w[c];
      dv[c] = tangle->vels[k].p[c] - tangle->vels[l].p[c];
    }
    double dot = 0;
    for (int c = 0; c < 3; ++c) dot += dx[c] * dv[c];
    if (dot > 0) continue;
    const int knext = tangle->connections[k].forward, kprev = tangle->connections[k].reverse;
    const int lnext = tangle->connections[l].forward, lprev = tangle->connections[l].reverse;
    int changed[4];
    if (!do_reconnection(tangle, k, l, changed)) continue;
    // the same links on the device
    for (int c = 0; c < 4; ++c) {
      const int m = changed[c];
      if (!ov_cuda_ok(cudaMemcpyAsync(R.s.links.as<int2>() + m, &tangle->connections[m], sizeof(int2),
                                      cudaMemcpyHostToDevice, R.s.stream),
                      "cudaMemcpyAsync"))
        return -ov_last_error();
    }
    const int flag[10] = {k, tangle->connections[k].forward, tangle->connections[k].reverse, knext, kprev,
                          l, tangle->connections[l].forward, tangle->connections[l].reverse, lnext, lprev};
    for (int f : flag) tangle->recalculate[f]++;
    ++nrecs;
    done_k = k;
  }
  if (!ov_cuda_ok(cudaStreamSynchronize(R.s.stream), "cudaStreamSynchronize")) return -ov_last_error();
  return nrecs;
}

}  // extern "C"
