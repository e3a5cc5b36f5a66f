// ov_remesh.cu - remesh (src/tangle.c:824-873) and enforce_boundaries
// (src/tangle.c:796-819) with the O(N) work on the GPU.
//
// The reference visits the slots in order.  At each node it may remove the
// node, merging it into a neighbour (remove_point, src/tangle.c:1017-1066),
// or add a node after it (add_point, src/tangle.c:1069-1150); after every
// change it recomputes the segment lengths, tangents and normals of the
// whole tangle.  A node's decision reads only its own and its reverse
// neighbour's segment length and the links around it.  A change moves at
// most one node and relinks at most three, so it alters segment lengths
// within one link and tangents and normals within six links (the 4-point
// stencils reach four links; next to a pinned node they also read the
// neighbours' tangents).  Every other value stays what it was, so the pass
// reduces to:
//   GPU   one scan of all nodes for those whose decision is a change;
//   host  the reference's loop over those nodes and the nodes near earlier
//         changes, in slot order, with the segment lengths near each change
//         recomputed at once in the reference's operations;
//   GPU   tangents and normals of the nodes near changes, recomputed when a
//         later change reads one of them and once at the end;
//   GPU   enforce_boundaries over all nodes when nodes were added.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <queue>
#include <vector>

#include "ov_internal.h"
#include "ov_links.cuh"

namespace {

constexpr int kThreads = 256;

// Nodes whose remesh decision is a change (the tests of src/tangle.c:839-865
// on the stored segment lengths), appended to cand (bounded by cap).
__global__ void k_remesh_scan(Links L, const double* __restrict__ dxi, int n, double min_dist,
                              double max_dist, int* cand, int cap, int* count, int* flag) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n || L.st[k].x == OV_EMPTY) return;
  const int2 lk = L.lk[k];
  const int next = lk.x, prev = lk.y;
  double lf = 0, lr = 0;
  if (next >= 0 && !arc_length(L, dxi, k, 1, lf)) { atomicOr(flag, 1); return; }
  if (prev >= 0 && !arc_length(L, dxi, k, -1, lr)) { atomicOr(flag, 1); return; }
  const bool remove = next >= 0 && prev >= 0 && !(L.lk[prev].y < 0 && L.lk[next].x < 0) &&
                      ((lf < min_dist || lr < min_dist) && (lf + lr) < max_dist);
  const bool add = next >= 0 && lf > max_dist;
  if (remove || add) {
    const int slot = atomicAdd(count, 1);
    if (slot < cap) cand[slot] = k;
  }
}

// A node's position, links and status as the host has them after a change.
struct NodePatch {
  double p[3];
  int slot, fwd, rev, status, pin, pad;
};
static_assert(sizeof(NodePatch) == 48, "NodePatch layout");

__global__ void k_patch(const NodePatch* __restrict__ np, int n, double* pos, int2* links, int2* status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const NodePatch q = np[i];
  st3(pos, q.slot, mk3(q.p[0], q.p[1], q.p[2]));
  links[q.slot] = make_int2(q.fwd, q.rev);
  status[q.slot] = make_int2(q.status, q.pin);
}

// dxi, tangent and normal of the slots idx[0 .. n-1], 7 doubles each
__global__ void k_gather_geom(const int* __restrict__ idx, int n, const double* __restrict__ dxi,
                              const double* __restrict__ tan, const double* __restrict__ nrm, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k = idx[i];
  double* o = out + 7 * (size_t)i;
  o[0] = dxi[k];
  const d3 t = ld3(tan, k), m = ld3(nrm, k);
  o[1] = t.x; o[2] = t.y; o[3] = t.z;
  o[4] = m.x; o[5] = m.y; o[6] = m.z;
}

struct BoxFaces {
  double lo[3], hi[3], L[3];
  int periodic_face[6];   // wall[face] == WALL_PERIODIC, faces X_L .. Z_H
};

// enforce_boundaries: a node outside the box through a periodic face moves
// by one box length until it is inside (out_of_box, src/tangle.c:766-794:
// the last of the six face tests that fails names the face, and only a
// periodic face moves the node; periodic_shift, src/vec3_maths.c:155-200).
// Moved slots are appended to moved; a node still outside after 64 moves
// sets flag bit 4.
__global__ void k_enforce(BoxFaces B, const int2* __restrict__ status, double* pos, int n, int* moved,
                          int* count, int* flag) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n || status[k].x == OV_EMPTY) return;
  double p[3] = {pos[3 * (size_t)k], pos[3 * (size_t)k + 1], pos[3 * (size_t)k + 2]};
  bool changed = false;
  int it = 0;
  for (; it < 64; ++it) {
    int face = -1;
    for (int c = 0; c < 3; ++c) {
      if (p[c] < B.lo[c]) face = 2 * c;
      if (p[c] > B.hi[c]) face = 2 * c + 1;
    }
    if (face > -1 && !B.periodic_face[face]) face = -1;
    if (face < 0) break;
    const int c = face >> 1;
    p[c] = (face & 1) ? __dsub_rn(p[c], B.L[c]) : __dadd_rn(p[c], B.L[c]);
    changed = true;
  }
  if (it == 64) atomicOr(flag, 4);
  if (changed) {
    pos[3 * (size_t)k] = p[0];
    pos[3 * (size_t)k + 1] = p[1];
    pos[3 * (size_t)k + 2] = p[2];
    moved[atomicAdd(count, 1)] = k;
  }
}

__global__ void k_gather_pos(const int* __restrict__ idx, int n, const double* __restrict__ pos, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const d3 p = ld3(pos, idx[i]);
  st3(out, i, p);
}

int blocks_for(int n) { return (n + kThreads - 1) / kThreads; }

// ---------------------------------------------------------------- host side
// Host restatements of the reference's vector steps, in its operation order
// (src/vec3_maths.c: vec3_add / vec3_sub / vec3_mul component by component,
// vec3_d as sqrt(((0 + x x) + y y) + z z)).
inline double h_norm(const double v[3]) {
  double s = 0;
  for (int c = 0; c < 3; ++c) s += v[c] * v[c];
  return sqrt(s);
}

// seg_pwrap (src/vec3_maths.c:105-138): r2 moved by one box length per
// periodic axis when it is more than half a box from r1
inline void h_pwrap(const tangle_state* t, const double* r1, const double* r2, double* out) {
  for (int c = 0; c < 3; ++c) {
    out[c] = r2[c];
    if (t->box.wall[2 * c] != WALL_PERIODIC) continue;
    const double L = t->box.top_right_front.p[c] - t->box.bottom_left_back.p[c];
    const double d = r2[c] - r1[c];
    if (d > L * 0.5) out[c] = r2[c] - L;
    else if (d < -L * 0.5) out[c] = r2[c] + L;
  }
}

inline bool h_pinned(int st) { return st == PINNED || st == PINNED_SLIP; }

// The stored segment length of node k as update_tangent_normal leaves it:
// the distance to the next node after the periodic wrap; at a pinned end
// without a forward link, to the mirror image of the reverse neighbour in
// the pinning wall (the device's k_dxi, step_node one link forward).
bool h_dxi(const tangle_state* t, int k, double& out) {
  const double* s0 = t->vnodes[k].p;
  double s1[3];
  const int f = t->connections[k].forward;
  if (f >= 0) {
    for (int c = 0; c < 3; ++c) s1[c] = t->vnodes[f].p[c];
  } else {
    const int r = t->connections[k].reverse;
    if (!h_pinned(t->status[k].status) || r < 0) return false;
    const int face = t->status[k].pin_wall;
    if (face < 0 || face > 5) return false;
    for (int c = 0; c < 3; ++c) s1[c] = t->vnodes[r].p[c];
    const int c = face >> 1;
    const double wp = (face & 1) ? t->box.top_right_front.p[c] : t->box.bottom_left_back.p[c];
    s1[c] = 2.0 * wp - s1[c];
  }
  double w[3], d[3];
  h_pwrap(t, s0, s1, w);
  for (int c = 0; c < 3; ++c) d[c] = s0[c] - w[c];
  out = h_norm(d);
  return true;
}

// arc_length (src/tangle.c:208-243) for one link forward (dist = 1) or
// back (dist = -1): the stored segment length, turning back at a pinned end
bool h_arc(const tangle_state* t, int k, int dist, double& out) {
  double acc = 0;
  int cur = k, d = dist;
  for (int it = 0; it < 16 && d != 0; ++it) {
    if (t->status[cur].status == EMPTY) return false;
    const bool pin = h_pinned(t->status[cur].status);
    const int f = t->connections[cur].forward, r = t->connections[cur].reverse;
    if (d > 0) {
      if (f < 0) {
        if (!pin) return false;
        d = -d;
        continue;
      }
      acc += t->dxi[cur];
      cur = f;
      --d;
    } else {
      if (r < 0) {
        if (!pin) return false;
        d = -d;
        continue;
      }
      acc += t->dxi[r];
      cur = r;
      ++d;
    }
  }
  if (d != 0) return false;
  out = acc;
  return true;
}

struct RemeshState {
  ov_state_impl s;
  DevBuf cand, count, patch, list, gather, moved;
  char* stage = nullptr;   // pinned host staging
  size_t stage_bytes = 0;
  ~RemeshState() {
    if (stage) cudaFreeHost(stage);
  }
  bool reserve_stage(size_t bytes) {
    if (bytes <= stage_bytes) return true;
    if (stage) cudaFreeHost(stage);
    stage = nullptr;
    stage_bytes = 0;
    const size_t want = std::max(bytes, 2 * stage_bytes + 4096);
    if (!ov_cuda_ok(cudaMallocHost(&stage, want), "cudaMallocHost")) return false;
    stage_bytes = want;
    return true;
  }
};

RemeshState& remesh_state() {
  static thread_local RemeshState r;
  return r;
}

// The pass over one tangle.
class Pass {
 public:
  Pass(RemeshState& R, tangle_state* t, double min_dist, double max_dist, ov_expand_fn expand)
      : R_(R), s_(&R.s), t_(t), min_(min_dist), max_(max_dist), expand_(expand) {}

  int run() {
    if (!upload_all()) return -ov_last_error();
    std::vector<int> cand;
    if (!scan(cand)) return -ov_last_error();
    resize_host();
    for (int k : cand) heap_.push(k);
    int changes = 0, added = 0, cur = -1;
    while (!heap_.empty()) {
      const int k = heap_.top();
      heap_.pop();
      if (k <= cur) continue;
      cur = k;
      if (k >= t_->N || t_->status[k].status == EMPTY) continue;
      const int next = t_->connections[k].forward, prev = t_->connections[k].reverse;
      double lf = 0, lr = 0;
      if ((next >= 0 && !h_arc(t_, k, 1, lf)) || (prev >= 0 && !h_arc(t_, k, -1, lr))) {
        ov_set_error(OV_ERR_INVALID, "remesh: broken vortex links at node %d", k);
        return -OV_ERR_INVALID;
      }
      if (next >= 0 && prev >= 0 &&
          !(t_->connections[prev].reverse < 0 && t_->connections[next].forward < 0) &&
          ((lf < min_ || lr < min_) && (lf + lr) < max_)) {
        if (!remove_point(k, lf < min_ ? +1 : -1)) return -ov_last_error();
        ++changes;
      }
      if (next >= 0 && lf > max_) {
        // (a removal needs lf + lr < max_dist, so at most one of the two runs)
        if (!add_point(k)) return -ov_last_error();
        ++changes;
        ++added;
      }
    }
    if (!flush()) return -ov_last_error();
    if (added && !enforce()) return -ov_last_error();
    return changes;
  }

  // enforce_boundaries on the device copy; moved positions back to the host
  bool enforce() {
    const int n = t_->N;
    if (n == 0) return true;
    BoxFaces B;
    for (int c = 0; c < 3; ++c) {
      B.lo[c] = t_->box.bottom_left_back.p[c];
      B.hi[c] = t_->box.top_right_front.p[c];
      B.L[c] = t_->box.top_right_front.p[c] - t_->box.bottom_left_back.p[c];
    }
    for (int f = 0; f < 6; ++f) B.periodic_face[f] = t_->box.wall[f] == WALL_PERIODIC;
    if (!R_.moved.reserve(sizeof(int) * (size_t)n) || !R_.count.reserve(sizeof(int)) ||
        !R_.gather.reserve(sizeof(double) * 3 * (size_t)n))
      return false;
    int* flag = s_->dflag.as<int>();
    OV_TRY_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s_->stream));
    OV_TRY_CUDA(cudaMemsetAsync(R_.count.p, 0, sizeof(int), s_->stream));
    k_enforce<<<blocks_for(n), kThreads, 0, s_->stream>>>(B, s_->status.as<int2>(), s_->pos.as<double>(), n,
                                                           R_.moved.as<int>(), R_.count.as<int>(), flag);
    OV_LAUNCHED();
    OV_TRY_CUDA(cudaGetLastError());
    int h[2] = {0, 0};
    OV_TRY_CUDA(cudaMemcpyAsync(&h[0], R_.count.p, sizeof(int), cudaMemcpyDeviceToHost, s_->stream));
    OV_TRY_CUDA(cudaMemcpyAsync(&h[1], flag, sizeof(int), cudaMemcpyDeviceToHost, s_->stream));
    OV_TRY_CUDA(cudaStreamSynchronize(s_->stream));
    if (h[1] & 4) {
      ov_set_error(OV_ERR_INVALID, "enforce_boundaries: a node is more than 64 box lengths outside the box");
      return false;
    }
    const int m = h[0];
    moved_ = m;
    if (m == 0) return true;
    k_gather_pos<<<blocks_for(m), kThreads, 0, s_->stream>>>(R_.moved.as<int>(), m, s_->pos.as<double>(),
                                                               R_.gather.as<double>());
    OV_LAUNCHED();
    OV_TRY_CUDA(cudaGetLastError());
    if (!R_.reserve_stage((sizeof(int) + 3 * sizeof(double)) * (size_t)m)) return false;
    double* hp = reinterpret_cast<double*>(R_.stage);
    int* hi = reinterpret_cast<int*>(R_.stage + 3 * sizeof(double) * (size_t)m);
    OV_TRY_CUDA(cudaMemcpyAsync(hp, R_.gather.p, 3 * sizeof(double) * (size_t)m, cudaMemcpyDeviceToHost,
                                s_->stream));
    OV_TRY_CUDA(cudaMemcpyAsync(hi, R_.moved.p, sizeof(int) * (size_t)m, cudaMemcpyDeviceToHost, s_->stream));
    OV_TRY_CUDA(cudaStreamSynchronize(s_->stream));
    for (int i = 0; i < m; ++i)
      for (int c = 0; c < 3; ++c) t_->vnodes[hi[i]].p[c] = hp[3 * i + c];
    return true;
  }

  bool upload_positions_status() { return ov_upload_tangle(s_, t_); }
  int moved() const { return moved_; }

 private:
  // positions, links and status, and the stored geometry as the caller has it
  bool upload_all() {
    if (!ov_upload_tangle(s_, t_)) return false;
    const size_t n = (size_t)t_->N;
    if (n == 0) return true;
    OV_TRY_CUDA(cudaMemcpyAsync(s_->dxi.p, t_->dxi, sizeof(double) * n, cudaMemcpyHostToDevice, s_->stream));
    OV_TRY_CUDA(cudaMemcpyAsync(s_->tan.p, t_->tangents, 24 * n, cudaMemcpyHostToDevice, s_->stream));
    OV_TRY_CUDA(cudaMemcpyAsync(s_->nrm.p, t_->normals, 24 * n, cudaMemcpyHostToDevice, s_->stream));
    return true;
  }

  bool scan(std::vector<int>& out) {
    const int n = t_->N;
    out.clear();
    if (n == 0) return true;
    int cap = std::max(1024, n / 16);
    int* flag = s_->dflag.as<int>();
    for (int attempt = 0; attempt < 2; ++attempt) {
      if (!R_.cand.reserve(sizeof(int) * (size_t)cap) || !R_.count.reserve(sizeof(int))) return false;
      OV_TRY_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s_->stream));
      OV_TRY_CUDA(cudaMemsetAsync(R_.count.p, 0, sizeof(int), s_->stream));
      k_remesh_scan<<<blocks_for(n), kThreads, 0, s_->stream>>>(Links{s_->links.as<int2>(), s_->status.as<int2>()},
                                                                 s_->dxi.as<double>(), n, min_, max_,
                                                                 R_.cand.as<int>(), cap, R_.count.as<int>(), flag);
      OV_LAUNCHED();
      OV_TRY_CUDA(cudaGetLastError());
      int h[2] = {0, 0};
      OV_TRY_CUDA(cudaMemcpyAsync(&h[0], R_.count.p, sizeof(int), cudaMemcpyDeviceToHost, s_->stream));
      OV_TRY_CUDA(cudaMemcpyAsync(&h[1], flag, sizeof(int), cudaMemcpyDeviceToHost, s_->stream));
      OV_TRY_CUDA(cudaStreamSynchronize(s_->stream));
      if (!ov_flag_status(h[1], "remesh")) return false;
      if (h[0] <= cap) {
        out.resize(h[0]);
        if (h[0])
          OV_TRY_CUDA(cudaMemcpy(out.data(), R_.cand.p, sizeof(int) * (size_t)h[0], cudaMemcpyDeviceToHost));
        std::sort(out.begin(), out.end());
        return true;
      }
      cap = h[0];
    }
    ov_set_error(OV_ERR_CUDA, "remesh: candidate count changed between two scans");
    return false;
  }

  void resize_host() {
    const size_t n = (size_t)t_->N;
    dirty_.assign(n, 0);
    patched_.assign(n, 0);
    stamp_.assign(n, 0);
    gen_ = 0;
    empty_.assign((n + 63) / 64, 0);
    for (size_t k = 0; k < n; ++k)
      if (t_->status[k].status == EMPTY) empty_[k >> 6] |= 1ULL << (k & 63);
  }

  // nodes within `radius` links of the seeds (the seeds included)
  void ball(const int* seeds, int ns, int radius, std::vector<int>& out) {
    out.clear();
    if (++gen_ == 0) {
      std::fill(stamp_.begin(), stamp_.end(), 0);
      gen_ = 1;
    }
    for (int i = 0; i < ns; ++i) {
      const int q = seeds[i];
      if (q < 0 || stamp_[q] == gen_) continue;
      stamp_[q] = gen_;
      out.push_back(q);
    }
    size_t lo = 0;
    for (int r = 0; r < radius; ++r) {
      const size_t hi = out.size();
      for (size_t i = lo; i < hi; ++i) {
        const int q = out[i];
        const int nb[2] = {t_->connections[q].forward, t_->connections[q].reverse};
        for (int j : nb)
          if (j >= 0 && stamp_[j] != gen_) {
            stamp_[j] = gen_;
            out.push_back(j);
          }
      }
      lo = hi;
    }
  }

  void mark_patched(int k) {
    if (!patched_[k]) {
      patched_[k] = 1;
      patch_list_.push_back(k);
    }
  }

  // After a change at the seeds: exact segment lengths within two links,
  // stale tangents and normals within six, decisions to revisit within
  // three (those after slot k, which the loop has not reached).
  bool after_change(const int* seeds, int ns, int k) {
    std::vector<int> near;
    ball(seeds, ns, 2, near);
    for (int q : near) {
      if (t_->status[q].status == EMPTY) continue;
      double d;
      if (!h_dxi(t_, q, d)) {
        ov_set_error(OV_ERR_INVALID, "remesh: broken vortex links at node %d", q);
        return false;
      }
      t_->dxi[q] = d;
    }
    ball(seeds, ns, 3, near);
    for (int q : near)
      if (q > k) heap_.push(q);
    ball(seeds, ns, 6, near);
    for (int q : near)
      if (!dirty_[q]) {
        dirty_[q] = 1;
        dirty_list_.push_back(q);
      }
    return true;
  }

  // recompute the stale tangents and normals on the device (after sending it
  // the changed nodes) and bring them and the segment lengths back
  bool flush() {
    std::vector<int> live;
    for (int q : dirty_list_) {
      dirty_[q] = 0;
      if (t_->status[q].status != EMPTY) live.push_back(q);
    }
    dirty_list_.clear();
    const int np = (int)patch_list_.size(), nd = (int)live.size();
    if (np == 0 && nd == 0) return true;
    const size_t patch_bytes = sizeof(NodePatch) * (size_t)np, list_bytes = sizeof(int) * (size_t)nd;
    const size_t list_off = (patch_bytes + 255) & ~(size_t)255;
    const size_t out_off = (list_off + list_bytes + 255) & ~(size_t)255;
    const size_t out_bytes = 7 * sizeof(double) * (size_t)nd;
    if (!R_.reserve_stage(out_off + out_bytes) || !R_.patch.reserve(out_off) ||
        !R_.gather.reserve(std::max<size_t>(out_bytes, 8)))
      return false;
    NodePatch* hp = reinterpret_cast<NodePatch*>(R_.stage);
    for (int i = 0; i < np; ++i) {
      const int q = patch_list_[i];
      patched_[q] = 0;
      NodePatch& e = hp[i];
      for (int c = 0; c < 3; ++c) e.p[c] = t_->vnodes[q].p[c];
      e.slot = q;
      e.fwd = t_->connections[q].forward;
      e.rev = t_->connections[q].reverse;
      e.status = t_->status[q].status;
      e.pin = t_->status[q].pin_wall;
      e.pad = 0;
    }
    patch_list_.clear();
    int* hl = reinterpret_cast<int*>(R_.stage + list_off);
    std::copy(live.begin(), live.end(), hl);
    OV_TRY_CUDA(cudaMemcpyAsync(R_.patch.p, R_.stage, list_off + list_bytes, cudaMemcpyHostToDevice, s_->stream));
    if (np) {
      k_patch<<<blocks_for(np), kThreads, 0, s_->stream>>>(R_.patch.as<NodePatch>(), np, s_->pos.as<double>(),
                                                            s_->links.as<int2>(), s_->status.as<int2>());
      OV_LAUNCHED();
    }
    if (nd) {
      const int* dl = reinterpret_cast<const int*>(static_cast<char*>(R_.patch.p) + list_off);
      int* flag = s_->dflag.as<int>();
      OV_TRY_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s_->stream));
      if (!ov_launch_geometry_list(s_->stream, s_->P, s_->links.as<int2>(), s_->status.as<int2>(),
                                   s_->pos.as<double>(), s_->dxi.as<double>(), s_->tan.as<double>(),
                                   s_->nrm.as<double>(), dl, nd, flag))
        return false;
      k_gather_geom<<<blocks_for(nd), kThreads, 0, s_->stream>>>(dl, nd, s_->dxi.as<double>(),
                                                                  s_->tan.as<double>(), s_->nrm.as<double>(),
                                                                  R_.gather.as<double>());
      OV_LAUNCHED();
      OV_TRY_CUDA(cudaGetLastError());
      double* ho = reinterpret_cast<double*>(R_.stage + out_off);
      int h = 0;
      OV_TRY_CUDA(cudaMemcpyAsync(ho, R_.gather.p, out_bytes, cudaMemcpyDeviceToHost, s_->stream));
      OV_TRY_CUDA(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, s_->stream));
      OV_TRY_CUDA(cudaStreamSynchronize(s_->stream));
      if (!ov_flag_status(h, "remesh (update_tangents_normals)")) return false;
      for (int i = 0; i < nd; ++i) {
        const int q = live[i];
        const double* o = ho + 7 * (size_t)i;
        t_->dxi[q] = o[0];
        for (int c = 0; c < 3; ++c) {
          t_->tangents[q].p[c] = o[1 + c];
          t_->normals[q].p[c] = o[4 + c];
        }
      }
    } else {
      OV_TRY_CUDA(cudaGetLastError());
      OV_TRY_CUDA(cudaStreamSynchronize(s_->stream));
    }
    ++flushes_;
    return true;
  }

  // search_next_free (src/tangle.c:729-745): next_free if that slot is
  // empty, else the first empty slot
  int next_free() {
    if (t_->next_free >= 0 && t_->next_free < t_->N && t_->status[t_->next_free].status == EMPTY)
      return t_->next_free++;
    for (size_t w = 0; w < empty_.size(); ++w)
      if (empty_[w]) {
        const int k = (int)(w * 64 + __builtin_ctzll(empty_[w]));
        if (k >= t_->N) break;
        t_->next_free = k + 1;
        return k;
      }
    return -1;
  }

  // get_tangle_next_free (src/tangle.c:747-756): with no empty slot the
  // caller's expand_tangle doubles the tangle, and the device copy follows
  bool take_slot(int& slot) {
    slot = next_free();
    if (slot >= 0) return true;
    if (!expand_) {
      ov_set_error(OV_ERR_INVALID,
                   "remesh: no empty slot for a new node (leave EMPTY slots or pass expand_tangle)");
      return false;
    }
    if (!flush()) return false;   // host copy complete before it is reallocated
    const int old_n = t_->N;
    expand_(t_, 2 * (size_t)std::max(old_n, 1));
    if (t_->N <= old_n) {
      ov_set_error(OV_ERR_INVALID, "remesh: expand_tangle did not grow the tangle");
      return false;
    }
    if (!upload_all()) return false;
    const size_t n = (size_t)t_->N;
    dirty_.resize(n, 0);
    patched_.resize(n, 0);
    stamp_.resize(n, 0);
    empty_.assign((n + 63) / 64, 0);
    for (size_t k = 0; k < n; ++k)
      if (t_->status[k].status == EMPTY) empty_[k >> 6] |= 1ULL << (k & 63);
    slot = next_free();
    if (slot < 0) {
      ov_set_error(OV_ERR_INVALID, "remesh: no empty slot after expand_tangle");
      return false;
    }
    return true;
  }

  bool need_fresh(int a, int b) {
    if ((a >= 0 && dirty_[a]) || (b >= 0 && dirty_[b])) return flush();
    return true;
  }

  // remove_point (src/tangle.c:1017-1066) with a merge direction
  bool remove_point(int k, int dir) {
    const int prev = t_->connections[k].reverse, next = t_->connections[k].forward;
    const int other = dir > 0 ? next : prev;
    if (t_->status[other].status == FREE) {
      if (!need_fresh(k, other)) return false;
      const double l = dir > 0 ? t_->dxi[k] : -t_->dxi[prev];
      const double* s0 = t_->vnodes[k].p;
      const double* s0p = t_->tangents[k].p;
      const double* s0pp = t_->normals[k].p;
      const double* s1 = t_->vnodes[other].p;
      const double* s1p = t_->tangents[other].p;
      const double* s1pp = t_->normals[other].p;
      double nw[3], a[3];
      for (int c = 0; c < 3; ++c) a[c] = s0[c] + s1[c];
      for (int c = 0; c < 3; ++c) nw[c] = a[c] * 0.5;
      for (int c = 0; c < 3; ++c) a[c] = s0p[c] - s1p[c];
      const double h = l / 2;
      for (int c = 0; c < 3; ++c) a[c] = a[c] * h;
      for (int c = 0; c < 3; ++c) nw[c] = nw[c] + a[c];
      for (int c = 0; c < 3; ++c) a[c] = s0pp[c] + s1pp[c];
      const double q = l * l / 16.0;
      for (int c = 0; c < 3; ++c) a[c] = a[c] * q;
      for (int c = 0; c < 3; ++c) nw[c] = nw[c] + a[c];
      for (int c = 0; c < 3; ++c) t_->vnodes[other].p[c] = nw[c];
    }
    if (prev >= 0) t_->connections[prev].forward = next;
    if (next >= 0) t_->connections[next].reverse = prev;
    t_->connections[k].forward = t_->connections[k].reverse = -1;
    t_->status[k].status = EMPTY;
    empty_[k >> 6] |= 1ULL << (k & 63);
    mark_patched(k);
    if (prev >= 0) mark_patched(prev);
    if (next >= 0) mark_patched(next);
    const int seeds[2] = {prev, next};
    return after_change(seeds, 2, k);
  }

  // add_point (src/tangle.c:1069-1150): a node between p and its forward
  // neighbour, on the circle through both with the mean curvature when that
  // is resolved, else at their midpoint
  bool add_point(int p) {
    const int next = t_->connections[p].forward;
    if (!need_fresh(p, next)) return false;
    int nw;
    if (!take_slot(nw)) return false;
    t_->status[nw].status = FREE;
    t_->status[nw].pin_wall = NOT_A_FACE;
    const double* s0 = t_->vnodes[p].p;
    double s1[3];
    h_pwrap(t_, s0, t_->vnodes[next].p, s1);
    const double* s0pp = t_->normals[p].p;
    const double* s1pp = t_->normals[next].p;
    double n[3], a[3], b[3], out[3];
    for (int c = 0; c < 3; ++c) n[c] = s0pp[c] + s1pp[c];
    for (int c = 0; c < 3; ++c) n[c] = n[c] * 0.5;
    const double nd = h_norm(n);
    const double lf = t_->dxi[p];
    if (nd < s_->P.max_curv / s_->P.dl_max && nd > 1e-8) {
      const double R = 1 / h_norm(n);
      const double dR = R * R - lf * lf / 4;
      const double delta = dR > 0 ? R - sqrt(dR) : R;
      const double inv = 1 / h_norm(n);
      for (int c = 0; c < 3; ++c) n[c] = n[c] * inv;
      for (int c = 0; c < 3; ++c) n[c] = n[c] * -1;
      for (int c = 0; c < 3; ++c) a[c] = s0[c] + s1[c];
      for (int c = 0; c < 3; ++c) a[c] = a[c] * 0.5;
      for (int c = 0; c < 3; ++c) b[c] = n[c] * delta;
      for (int c = 0; c < 3; ++c) out[c] = a[c] + b[c];
    } else {
      for (int c = 0; c < 3; ++c) out[c] = s0[c] + s1[c];
      for (int c = 0; c < 3; ++c) out[c] = out[c] * 0.5;
    }
    for (int c = 0; c < 3; ++c) t_->vnodes[nw].p[c] = out[c];
    t_->connections[nw].reverse = p;
    t_->connections[nw].forward = next;
    t_->connections[p].forward = nw;
    t_->connections[next].reverse = nw;
    empty_[nw >> 6] &= ~(1ULL << (nw & 63));
    mark_patched(nw);
    mark_patched(p);
    mark_patched(next);
    const int seeds[1] = {nw};
    return after_change(seeds, 1, p);
  }

  RemeshState& R_;
  ov_state_impl* s_;
  tangle_state* t_;
  double min_, max_;
  ov_expand_fn expand_;
  std::priority_queue<int, std::vector<int>, std::greater<int>> heap_;
  std::vector<char> dirty_, patched_;
  std::vector<int> dirty_list_, patch_list_;
  std::vector<unsigned> stamp_;
  unsigned gen_ = 0;
  std::vector<unsigned long long> empty_;
  int flushes_ = 0, moved_ = 0;
};

bool check_tangle(const tangle_state* t, const char* where, bool geometry) {
  if (!t || t->N < 0 || (t->N > 0 && (!t->vnodes || !t->connections || !t->status))) {
    ov_set_error(OV_ERR_INVALID, "%s: null tangle or arrays", where);
    return false;
  }
  if (geometry && t->N > 0 && (!t->dxi || !t->tangents || !t->normals)) {
    ov_set_error(OV_ERR_INVALID, "%s: the tangle's dxi, tangents and normals are needed", where);
    return false;
  }
  return true;
}

}  // namespace

extern "C" {

int ov_remesh(struct tangle_state* tangle, double min_dist, double max_dist, ov_expand_fn expand) {
  ov_clear_error();
  if (!check_tangle(tangle, "ov_remesh", true)) return -OV_ERR_INVALID;
  if (!(min_dist >= 0) || !(max_dist > 0)) {
    ov_set_error(OV_ERR_INVALID, "ov_remesh: min_dist and max_dist must be >= 0 and > 0");
    return -OV_ERR_INVALID;
  }
  if (!ov_ensure_init()) return -ov_last_error();
  Pass pass(remesh_state(), tangle, min_dist, max_dist, expand);
  return pass.run();
}

int ov_enforce_boundaries(struct tangle_state* tangle) {
  ov_clear_error();
  if (!check_tangle(tangle, "ov_enforce_boundaries", false)) return -OV_ERR_INVALID;
  if (!ov_ensure_init()) return -ov_last_error();
  Pass pass(remesh_state(), tangle, 0, 1, nullptr);
  if (!pass.upload_positions_status() || !pass.enforce()) return -ov_last_error();
  return pass.moved();
}

}  // extern "C"
