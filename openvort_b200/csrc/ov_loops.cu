// ov_loops.cu - eliminate_small_loops (src/tangle.c:876-943) on the GPU.
//
// The reference walks each vortex from its lowest unvisited slot and counts
// the steps around a closed loop, or out to both pinned ends of a line:
// either way one less than the vortex's node count.  A vortex with fewer
// steps than loop_length is deleted.  Before that, when switched on, it
// deletes loops lying wholly within a distance of the origin
// (src/tangle.c:945-972), within a distance of the z axis, or wholly
// beyond a distance from it (src/tangle.c:974-1015).  Every test is a
// property of a whole vortex, so here:
//   1. each node is labelled with the least slot of its vortex, by pointer
//      jumping along the forward and the reverse links (after r rounds a
//      node holds the least slot within 2^r links; the least of the two
//      directions covers a line, either one a closed loop);
//   2. per label, the node count and the AND of the radial tests;
//   3. the nodes of the vortices that fail are emptied and unlinked.
// The reference also leaves visit counts in tangle->recalculate; nothing
// reads them afterwards (reconnect zeroes them first) and they are not
// written here.
#include <climits>
#include <vector>

#include "ov_internal.h"

namespace {

constexpr int kThreads = 256;
int blocks_for(int n) { return (n + kThreads - 1) / kThreads; }

__global__ void k_lbl_init(const int2* __restrict__ links, const int2* __restrict__ status, int n, int* lab_f,
                           int* jmp_f, int* lab_b, int* jmp_b) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const bool live = status[k].x != OV_EMPTY;
  const int2 lk = links[k];
  lab_f[k] = lab_b[k] = live ? k : INT_MAX;
  jmp_f[k] = live ? lk.x : -1;
  jmp_b[k] = live ? lk.y : -1;
}

// one doubling round: the least label within twice the distance
__global__ void k_lbl_step(const int* __restrict__ lab, const int* __restrict__ jmp, int n, int* lab_out,
                           int* jmp_out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int j = jmp[k];
  if (j >= 0) {
    lab_out[k] = min(lab[k], lab[j]);
    jmp_out[k] = jmp[j];
  } else {
    lab_out[k] = lab[k];
    jmp_out[k] = -1;
  }
}

struct Cuts {
  int origin, zaxis, outer;
  double origin_cut, zaxis_cut, outer_cut;
};

// per vortex: node count and the AND of the three radial tests (bit 0:
// |r| < origin cut, vec3_d; bit 1: distance to the z axis < zaxis cut;
// bit 2: that distance > outer cut; Z_R of src/tangle.c:989)
__global__ void k_lbl_count(const int* __restrict__ lab_f, const int* __restrict__ lab_b,
                            const int2* __restrict__ status, const double* __restrict__ pos, int n, Cuts C,
                            int* size, unsigned* tests) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n || status[k].x == OV_EMPTY) return;
  const int l = min(lab_f[k], lab_b[k]);
  atomicAdd(&size[l], 1);
  if (C.origin | C.zaxis | C.outer) {
    const d3 p = ld3(pos, k);
    const double zr = __dsqrt_rn(__dadd_rn(__dmul_rn(p.x, p.x), __dmul_rn(p.y, p.y)));
    const unsigned bits = (norm_ref(p) < C.origin_cut ? 1u : 0u) | (zr < C.zaxis_cut ? 2u : 0u) |
                          (zr > C.outer_cut ? 4u : 0u);
    atomicAnd(&tests[l], bits);
  }
}

__global__ void k_lbl_kill(const int* __restrict__ lab_f, const int* __restrict__ lab_b, int n, Cuts C,
                           int loop_length, const int* __restrict__ size, const unsigned* __restrict__ tests,
                           int2* links, int2* status, int* killed, int* n_killed, int* n_vortices) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n || status[k].x == OV_EMPTY) return;
  const int l = min(lab_f[k], lab_b[k]);
  const unsigned t = tests[l];
  const bool kill = (C.origin && (t & 1u)) || (C.zaxis && (t & 2u)) || (C.outer && (t & 4u)) ||
                    size[l] - 1 < loop_length;
  if (!kill) return;
  links[k] = make_int2(-1, -1);
  status[k].x = OV_EMPTY;
  killed[atomicAdd(n_killed, 1)] = k;
  if (l == k) atomicAdd(n_vortices, 1);
}

struct LoopState {
  ov_state_impl s;
  DevBuf lab, jmp, size, tests, killed, counts;
};

LoopState& loop_state() {
  static thread_local LoopState r;
  return r;
}

// steps 1-3 on a state whose links and status (and positions, when a radial
// test is on) are current; the emptied slots are returned in out
bool eliminate(LoopState& R, int loop_length, std::vector<int>& out, int& vortices) {
  ov_state_impl* s = &R.s;
  const int n = s->n;
  out.clear();
  vortices = 0;
  if (n == 0) return true;
  const Cuts C{global_eliminate_origin_loops, global_eliminate_zaxis_loops, global_eliminate_outer_loops,
               global_eliminate_loops_origin_cutoff, global_eliminate_loops_zaxis_cutoff,
               global_eliminate_outer_loops_cutoff};
  const size_t nb = sizeof(int) * (size_t)n;
  if (!R.lab.reserve(4 * nb) || !R.jmp.reserve(4 * nb) || !R.size.reserve(nb) || !R.tests.reserve(nb) ||
      !R.killed.reserve(nb) || !R.counts.reserve(2 * sizeof(int)))
    return false;
  int* lab = R.lab.as<int>();
  int* jmp = R.jmp.as<int>();
  // [forward current, forward next, reverse current, reverse next]
  int* lf[2] = {lab, lab + n};
  int* jf[2] = {jmp, jmp + n};
  int* lb[2] = {lab + 2 * (size_t)n, lab + 3 * (size_t)n};
  int* jb[2] = {jmp + 2 * (size_t)n, jmp + 3 * (size_t)n};
  k_lbl_init<<<blocks_for(n), kThreads, 0, s->stream>>>(s->links.as<int2>(), s->status.as<int2>(), n, lf[0],
                                                         jf[0], lb[0], jb[0]);
  OV_LAUNCHED();
  int rounds = 1;
  while ((1LL << rounds) < n) ++rounds;
  int cur = 0;
  for (int r = 0; r < rounds; ++r) {
    k_lbl_step<<<blocks_for(n), kThreads, 0, s->stream>>>(lf[cur], jf[cur], n, lf[cur ^ 1], jf[cur ^ 1]);
    OV_LAUNCHED();
    k_lbl_step<<<blocks_for(n), kThreads, 0, s->stream>>>(lb[cur], jb[cur], n, lb[cur ^ 1], jb[cur ^ 1]);
    OV_LAUNCHED();
    cur ^= 1;
  }
  OV_TRY_CUDA(cudaMemsetAsync(R.size.p, 0, nb, s->stream));
  OV_TRY_CUDA(cudaMemsetAsync(R.tests.p, 0xff, nb, s->stream));
  OV_TRY_CUDA(cudaMemsetAsync(R.counts.p, 0, 2 * sizeof(int), s->stream));
  k_lbl_count<<<blocks_for(n), kThreads, 0, s->stream>>>(lf[cur], lb[cur], s->status.as<int2>(),
                                                          s->pos.as<double>(), n, C, R.size.as<int>(),
                                                          R.tests.as<unsigned>());
  OV_LAUNCHED();
  k_lbl_kill<<<blocks_for(n), kThreads, 0, s->stream>>>(lf[cur], lb[cur], n, C, loop_length, R.size.as<int>(),
                                                         R.tests.as<unsigned>(), s->links.as<int2>(),
                                                         s->status.as<int2>(), R.killed.as<int>(),
                                                         R.counts.as<int>(), R.counts.as<int>() + 1);
  OV_LAUNCHED();
  OV_TRY_CUDA(cudaGetLastError());
  int h[2] = {0, 0};
  OV_TRY_CUDA(cudaMemcpyAsync(h, R.counts.p, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
  OV_TRY_CUDA(cudaStreamSynchronize(s->stream));
  out.resize(h[0]);
  if (h[0]) OV_TRY_CUDA(cudaMemcpy(out.data(), R.killed.p, sizeof(int) * (size_t)h[0], cudaMemcpyDeviceToHost));
  vortices = h[1];
  return true;
}

}  // namespace

extern "C" {

int ov_eliminate_small_loops(struct tangle_state* tangle, int loop_length) {
  ov_clear_error();
  if (!tangle || tangle->N < 0 || (tangle->N > 0 && (!tangle->vnodes || !tangle->connections || !tangle->status))) {
    ov_set_error(OV_ERR_INVALID, "ov_eliminate_small_loops: null tangle or arrays");
    return -OV_ERR_INVALID;
  }
  LoopState& R = loop_state();
  if (!ov_upload_tangle(&R.s, tangle)) return -ov_last_error();
  std::vector<int> killed;
  int vortices = 0;
  if (!eliminate(R, loop_length, killed, vortices)) return -ov_last_error();
  for (int k : killed) {
    tangle->connections[k].forward = tangle->connections[k].reverse = -1;
    tangle->status[k].status = EMPTY;
  }
  return vortices;
}

}  // extern "C"
