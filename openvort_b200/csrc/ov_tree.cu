// ov_tree.cu - Barnes-Hut octree on the GPU, cell for cell the reference's
// geometric octree (octree_build / octree_inner_sort / make_child_box /
// octree_update_means, src/octree.c:21-272), built without recursion:
//
//  1. k_keys: each node descends from the domain box, recomputing the child
//     boxes with the reference's exact FP64 arithmetic and taking the first
//     child (in the reference's BLF..TRB order) that strictly contains it;
//     4 bits per level record the child (8 = contained by no child: the
//     reference drops such nodes from the subtree).  The descent stops at the
//     first box the walk treats as a leaf (min side < BH_grain) or the build
//     does not split (min side < BH_grain * dl_max).
//  2. LSD radix sort of the 128-bit keys (8 passes of 8 bits over the high
//     word, then ties ordered by the low word), stable, so nodes of one cell
//     keep slot order like the reference's node lists.
//  3. Karras radix tree over the sorted keys; every binary node whose range
//     is a whole cell at some level becomes an octree cell.  A cell that is
//     also its parent's only non-empty child (a chain) is kept once: the
//     opening test passes at the deepest level of the chain if it passes
//     anywhere in it, and the moments are the same.
//  4. Cells laid out in depth-first preorder (children in the reference's
//     order); each cell stores the index after its subtree (`skip`), which
//     lets the walk run without a stack.
//  5. Moments (centre of mass, total circulation, circulation tensor) summed
//     over each cell's own node range, as the reference does.
#include <float.h>

#include <algorithm>
#include <utility>

#include "ov_internal.h"

namespace {

constexpr int kMaxLevels = 32;
constexpr int kDigitDropped = 8;
enum { TERM_GRAIN = 0, TERM_BUILD = 1, TERM_DROP = 2 };

__device__ __forceinline__ double box_max(const double lo[3], const double hi[3]) {
  double a = __dsub_rn(hi[0], lo[0]), b = __dsub_rn(hi[1], lo[1]), c = __dsub_rn(hi[2], lo[2]);
  if (a > b) return a > c ? a : c;
  return b > c ? b : c;
}
__device__ __forceinline__ double box_min(const double lo[3], const double hi[3]) {
  double a = __dsub_rn(hi[0], lo[0]), b = __dsub_rn(hi[1], lo[1]), c = __dsub_rn(hi[2], lo[2]);
  if (a < b) return a < c ? a : c;
  return b < c ? b : c;
}

// Child box k of (plo, phi), exactly as make_child_box (src/octree.c:158-235).
//   k : 0 BLF  1 BLB  2 BRF  3 BRB  4 TLF  5 TLB  6 TRF  7 TRB
// Corner boxes are [lo, c] or [c, hi]; four children shift a corner box by
// half a side along one axis.
__device__ __forceinline__ void child_box(const double plo[3], const double phi[3], const double c[3],
                                          const double Lh[3], int k, int quad, double lo[3],
                                          double hi[3]) {
  const bool from_lo = (k == 0 || k == 1 || k == 3 || k == 5);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    lo[a] = from_lo ? plo[a] : c[a];
    hi[a] = from_lo ? c[a] : phi[a];
  }
  switch (k) {
    case 0: lo[0] = __dadd_rn(lo[0], Lh[0]); hi[0] = __dadd_rn(hi[0], Lh[0]); break;
    case 2: lo[2] = __dsub_rn(lo[2], Lh[2]); hi[2] = __dsub_rn(hi[2], Lh[2]); break;
    case 3: lo[1] = __dadd_rn(lo[1], Lh[1]); hi[1] = __dadd_rn(hi[1], Lh[1]); break;
    case 4: lo[1] = __dsub_rn(lo[1], Lh[1]); hi[1] = __dsub_rn(hi[1], Lh[1]); break;
    case 5: lo[2] = __dadd_rn(lo[2], Lh[2]); hi[2] = __dadd_rn(hi[2], Lh[2]); break;
    case 7: lo[0] = __dsub_rn(lo[0], Lh[0]); hi[0] = __dsub_rn(hi[0], Lh[0]); break;
    default: break;
  }
  if (quad) hi[2] = phi[2];
}

__device__ __forceinline__ void split_params(const double lo[3], const double hi[3], double c[3],
                                             double Lh[3]) {
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    c[a] = __dmul_rn(__dadd_rn(lo[a], hi[a]), 0.5);
    Lh[a] = __dsub_rn(hi[a], lo[a]) / 2;   // exact halving
  }
}

__device__ __forceinline__ int key_digit(uint64_t hi, uint64_t lo, int level) {
  // level 1 occupies the top 4 bits of hi; levels 17..32 are in lo
  if (level <= 16) return (int)((hi >> (64 - 4 * level)) & 15ull);
  return (int)((lo >> (64 - 4 * (level - 16))) & 15ull);
}

__device__ __forceinline__ void set_digit(uint64_t& hi, uint64_t& lo, int level, int d) {
  if (level <= 16) hi |= (uint64_t)d << (64 - 4 * level);
  else lo |= (uint64_t)d << (64 - 4 * (level - 16));
}

// ---------------------------------------------------------------- 1. keys
__global__ void k_keys(OvParams P, const double* __restrict__ pos, const int2* __restrict__ status,
                       int n, uint64_t* khi, uint64_t* klo, int* vals, int* term, int* counters) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  vals[k] = k;
  if (status[k].x == OV_EMPTY) {
    khi[k] = ~0ull;
    klo[k] = ~0ull;
    term[k] = -1;
    return;
  }
  atomicAdd(&counters[0], 1);
  const int nch = P.quadtree ? 4 : 8;
  const double px = pos[3 * k], py = pos[3 * k + 1], pz = pos[3 * k + 2];
  double lo[3] = {P.lo[0], P.lo[1], P.lo[2]}, hi[3] = {P.hi[0], P.hi[1], P.hi[2]};
  const double build_min = P.grain * P.dl_max;
  uint64_t h = 0, l = 0;
  int level = 0, tl = 0, tk = TERM_BUILD;
  for (;;) {
    double Lmin = box_min(lo, hi);
    if (Lmin < P.grain) { tl = level; tk = TERM_GRAIN; break; }
    if (Lmin < build_min) { tl = level; tk = TERM_BUILD; break; }
    if (level == kMaxLevels) { tl = level; tk = TERM_BUILD; atomicOr(&counters[1], 1); break; }
    double c[3], Lh[3];
    split_params(lo, hi, c, Lh);
    int digit = kDigitDropped;
    for (int ch = 0; ch < nch; ++ch) {
      double clo[3], chi[3];
      child_box(lo, hi, c, Lh, ch, P.quadtree, clo, chi);
      // strict containment (in_box, src/vec3_maths.c:67-77)
      if (px > clo[0] && px < chi[0] && py > clo[1] && py < chi[1] && pz > clo[2] && pz < chi[2]) {
        digit = ch;
#pragma unroll
        for (int a = 0; a < 3; ++a) { lo[a] = clo[a]; hi[a] = chi[a]; }
        break;
      }
    }
    ++level;
    set_digit(h, l, level, digit);
    if (digit == kDigitDropped) {
      tl = level - 1;
      tk = TERM_DROP;
      if (tl == 0) atomicAdd(&counters[3], 1);   // outside the root box
      break;
    }
  }
  khi[k] = h;
  klo[k] = l;
  term[k] = tl | (tk << 8);
  atomicMax(&counters[2], tl);
}

// ---------------------------------------------------------------- 2. sort
constexpr int kRsThreads = 256;
constexpr int kRsItems = 16;
constexpr int kRsTile = kRsThreads * kRsItems;

__global__ void k_rs_hist(const uint64_t* __restrict__ keys, int n, int shift, unsigned* hist,
                          int nblocks) {
  __shared__ unsigned h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  int base = blockIdx.x * kRsTile;
  for (int t = 0; t < kRsItems; ++t) {
    int i = base + t * kRsThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255], 1u);
  }
  __syncthreads();
  hist[threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of m unsigned values in three launches: the sum of each
// 1024-value block, a scan of those sums, then every block's own scan plus
// its offset.  Every access is one coalesced value per thread.
constexpr int kScanThreads = 1024;

// exclusive prefix of x over the block's threads (1024, 32 warps); the block
// total in `total`.  sh holds 33 values.
__device__ __forceinline__ unsigned block_excl_scan(unsigned x, unsigned* sh, unsigned& total) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned inc = x;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const unsigned y = __shfl_up_sync(FULL, inc, off);
    if (lane >= off) inc += y;
  }
  if (lane == 31) sh[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const unsigned w = sh[lane];
    unsigned wi = w;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const unsigned y = __shfl_up_sync(FULL, wi, off);
      if (lane >= off) wi += y;
    }
    sh[lane] = wi - w;
    if (lane == 31) sh[32] = wi;
  }
  __syncthreads();
  total = sh[32];
  const unsigned r = sh[warp] + inc - x;
  __syncthreads();   // sh is free again on return
  return r;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_sums(const unsigned* __restrict__ v, int m,
                                                            unsigned* sums) {
  __shared__ unsigned sh[33];
  const int i = blockIdx.x * kScanThreads + threadIdx.x;
  unsigned tot;
  block_excl_scan(i < m ? v[i] : 0u, sh, tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// one block: exclusive scan of nb block sums, 1024 at a time with a carry
__global__ void __launch_bounds__(kScanThreads) k_scan_top(unsigned* sums, int nb) {
  __shared__ unsigned sh[33];
  unsigned carry = 0;
  for (int b0 = 0; b0 < nb; b0 += kScanThreads) {
    const int i = b0 + threadIdx.x;
    unsigned tot;
    const unsigned e = block_excl_scan(i < nb ? sums[i] : 0u, sh, tot);
    if (i < nb) sums[i] = carry + e;
    carry += tot;
  }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_apply(unsigned* v, int m,
                                                             const unsigned* __restrict__ sums) {
  __shared__ unsigned sh[33];
  const int i = blockIdx.x * kScanThreads + threadIdx.x;
  const unsigned x = i < m ? v[i] : 0u;
  unsigned tot;
  const unsigned e = block_excl_scan(x, sh, tot);
  if (i < m) v[i] = sums[blockIdx.x] + e;
}

__global__ void k_rs_scatter(const uint64_t* __restrict__ kin, const int* __restrict__ vin,
                             uint64_t* kout, int* vout, int n, int shift,
                             const unsigned* __restrict__ hist, int nblocks) {
  __shared__ unsigned offs[256];
  __shared__ unsigned wcnt[kRsThreads / 32][256];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  offs[threadIdx.x] = hist[threadIdx.x * nblocks + blockIdx.x];
  for (int w = 0; w < kRsThreads / 32; ++w) wcnt[w][threadIdx.x] = 0;
  __syncthreads();
  int base = blockIdx.x * kRsTile;
  const unsigned lt_mask = (1u << lane) - 1u;
  for (int t = 0; t < kRsItems; ++t) {
    int i = base + t * kRsThreads + threadIdx.x;
    bool valid = i < n;
    uint64_t key = valid ? kin[i] : 0;
    int val = valid ? vin[i] : 0;
    int d = valid ? (int)((key >> shift) & 255) : 256;
    unsigned peers = __match_any_sync(0xffffffffu, d);
    unsigned rank_w = __popc(peers & lt_mask);
    if (valid && rank_w == 0) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    if (valid) {
      unsigned r = offs[d] + rank_w;
      for (int w = 0; w < warp; ++w) r += wcnt[w][d];
      kout[r] = key;
      vout[r] = val;
    }
    __syncthreads();
    unsigned tot = 0;
    for (int w = 0; w < kRsThreads / 32; ++w) {
      tot += wcnt[w][threadIdx.x];
      wcnt[w][threadIdx.x] = 0;
    }
    offs[threadIdx.x] += tot;
    __syncthreads();
  }
}

// gather the low key words and termination codes into sorted order
__global__ void k_gather_lo(const int* __restrict__ perm, const uint64_t* __restrict__ klo_slot,
                            const int* __restrict__ term_slot, uint64_t* klo, int* term, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int s = perm[i];
  klo[i] = klo_slot[s];
  term[i] = term_slot[s];
}

// order runs of equal high words by the low word (insertion sort; runs are
// nodes closer than 2^-16 of the box, essentially always length 1)
__global__ void k_fix_ties(const uint64_t* __restrict__ khi, uint64_t* klo, int* perm, int* term,
                           int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (i > 0 && khi[i - 1] == khi[i]) return;
  int e = i + 1;
  while (e < n && khi[e] == khi[i]) ++e;
  for (int a = i + 1; a < e; ++a) {
    uint64_t kl = klo[a];
    int pv = perm[a], tv = term[a];
    int b = a - 1;
    while (b >= i && klo[b] > kl) {
      klo[b + 1] = klo[b];
      perm[b + 1] = perm[b];
      term[b + 1] = term[b];
      --b;
    }
    klo[b + 1] = kl;
    perm[b + 1] = pv;
    term[b + 1] = tv;
  }
}

// ---------------------------------------------------------------- 3. radix tree
struct BNode {      // internal node of the binary radix tree
  int first, last;  // key range
  int delta;        // common prefix length in bits (ties: 128 + index bits)
  int left, right;  // child ids: internal i -> i, leaf i -> leaf_base + i
  int parent;       // internal parent, -1 for the root
  int pad0, pad1;
};

__device__ __forceinline__ int kdelta(const uint64_t* hi, const uint64_t* lo, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  uint64_t a = hi[i] ^ hi[j];
  if (a) return __clzll(a);
  uint64_t b = lo[i] ^ lo[j];
  if (b) return 64 + __clzll(b);
  return 128 + __clz(i ^ j);
}

__global__ void k_karras(const uint64_t* __restrict__ hi, const uint64_t* __restrict__ lo, int n,
                         BNode* nodes, int* leaf_parent) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  int d = (kdelta(hi, lo, n, i, i + 1) - kdelta(hi, lo, n, i, i - 1)) > 0 ? 1 : -1;
  int dmin = kdelta(hi, lo, n, i, i - d);
  int lmax = 2;
  while (kdelta(hi, lo, n, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t >= 1; t >>= 1)
    if (kdelta(hi, lo, n, i, i + (l + t) * d) > dmin) l += t;
  int j = i + l * d;
  int dn = kdelta(hi, lo, n, i, j);
  int s = 0, t = l;
  do {
    t = (t + 1) >> 1;
    if (kdelta(hi, lo, n, i, i + (s + t) * d) > dn) s += t;
  } while (t > 1);
  int gam = i + s * d + min(d, 0);
  int first = min(i, j), last = max(i, j);
  const int leaf_base = n - 1;
  int left = (first == gam) ? leaf_base + gam : gam;
  int right = (last == gam + 1) ? leaf_base + gam + 1 : gam + 1;
  BNode& nd = nodes[i];
  nd.first = first;
  nd.last = last;
  nd.delta = dn;
  nd.left = left;
  nd.right = right;
  if (left >= leaf_base) leaf_parent[left - leaf_base] = i; else nodes[left].parent = i;
  if (right >= leaf_base) leaf_parent[right - leaf_base] = i; else nodes[right].parent = i;
  if (i == 0) nd.parent = -1;
}

// ---------------------------------------------------------------- 4. cells
struct CellInfo {   // per binary node (internal ids first, then leaves)
  int is_cell;
  int ltop;         // first octree level at which the range is a whole cell
  int kind;         // CELL_*
  int mac_level;    // level whose box the opening test uses (-1: none)
  int lbot;         // last level of the chain (children start one below)
};

__device__ __forceinline__ void bnode_range(const BNode* nodes, int n, int b, int& first, int& last,
                                            int& dX, int& parent, const int* leaf_parent) {
  const int leaf_base = n - 1;
  if (b < leaf_base) {
    first = nodes[b].first;
    last = nodes[b].last;
    dX = nodes[b].delta;
    parent = nodes[b].parent;
  } else {
    first = last = b - leaf_base;
    dX = 1 << 20;
    parent = n > 1 ? leaf_parent[b - leaf_base] : -1;
  }
}

__global__ void k_classify(const BNode* __restrict__ nodes, const int* __restrict__ leaf_parent,
                           const int* __restrict__ term, int n, CellInfo* info, unsigned* cnt) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= 2 * n - 1) return;
  int first, last, dX, parent;
  bnode_range(nodes, n, b, first, last, dX, parent, leaf_parent);
  int dP = parent >= 0 ? nodes[parent].delta : -1;
  int ltop = (dP + 4) >> 2;
  int lbot = (b < n - 1) ? (dX >> 2) : (1 << 18);
  int tc = term[first];
  int tl = tc & 255, tk = tc >> 8;
  CellInfo ci;
  ci.ltop = ltop;
  ci.is_cell = ltop <= min(lbot, tl);
  ci.kind = CELL_LEAF1;
  ci.mac_level = -1;
  ci.lbot = ltop;
  if (ci.is_cell) {
    int N = last - first + 1;
    // the range ends its descent inside this chain: a stop is a property of
    // the shared box; a drop at level tl+1 is shared only when tl+1 <= lbot
    bool ends = (tk == TERM_DROP) ? (tl < lbot) : (tl <= lbot);
    if (N == 1) {
      ci.kind = CELL_LEAF1;
    } else if (ends) {
      if (tk == TERM_GRAIN) {
        if (tl == ltop) ci.kind = CELL_LEAFN;
        else { ci.kind = CELL_OPEN_P2P; ci.mac_level = tl - 1; }
      } else {  // unsplit (build stop) or every node dropped one level down
        ci.kind = CELL_OPEN_ZERO;
        ci.mac_level = tl;
      }
    } else {
      ci.kind = CELL_OPEN;
      ci.mac_level = lbot;
    }
    if (ci.kind != CELL_LEAF1) ci.lbot = ci.kind == CELL_OPEN_P2P ? tl : max(ci.mac_level, ltop);
    atomicAdd(&cnt[first], 1u);
  }
  info[b] = ci;
}

// Smallest s with fl(Lm / fl(sqrt(s))) < theta: the opening test of
// octree_get_vs (src/octree.c:296) as a threshold on the squared distance.
__device__ double mac_threshold(double Lm, double theta) {
  if (!(theta > 0)) return DBL_MAX;
  double s = (Lm / theta) * (Lm / theta);
  if (!(s > 0)) s = DBL_MIN;
  auto ok = [&](double x) { return __ddiv_rn(Lm, __dsqrt_rn(x)) < theta; };
  if (ok(s)) {
    for (int it = 0; it < 64; ++it) {
      double p = nextafter(s, 0.0);
      if (!(p > 0) || !ok(p)) break;
      s = p;
    }
  } else {
    for (int it = 0; it < 64 && !ok(s); ++it) s = nextafter(s, DBL_MAX);
  }
  return s;
}

// Rounding margin E of a cell's opening test for the multi-image walk: the
// walk decides all of a target's images from the target's own squared
// distance q0 when q0 >= thr + E (every image passes) or q0 < thr - E (every
// image fails, where no axis wraps).  Derivation, with u = 2^-53:
//   - the positions used are within [lo - L/4, hi + L/4] (walk targets are
//     checked; a non-root cell's centre of mass is a mean of nodes in the box),
//     so every FP64 value the wrapped distance forms (r -+ L, c -+ L, their
//     difference) is at most B = 3.5 max_a(|lo_a| + |hi_a|) in magnitude, and
//     each computed component differs from the exact r_a - c_a by at most
//     e = 4 u B;
//   - a computed squared distance q then differs from the exact Q by at most
//     D(Q) = (2 e sqrt(3 Q) + 3 e^2)(1 + 3.01 u) + 3.01 u Q (three roundings
//     of the squares and their sums);
//   - with E = 2 D(4 thr), q0 >= thr + E implies Q > thr + E/2, so each
//     image (whose exact distance is at least Q) computes q >= thr; q0 < thr - E
//     and equal exact distances imply each image computes q < thr.
// 1% slack covers the roundings of this formula and of thr -+ E; the value is
// rounded up to FP32.  Cells that never pass (thr = DBL_MAX) need no margin;
// a margin above thr / 2 disables both shortcuts (infinity).
__device__ float mac_margin(const OvParams& P, double thr) {
  if (thr == DBL_MAX) return 0.f;
  double B = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) B = fmax(B, fabs(P.lo[a]) + fabs(P.hi[a]));
  const double u = 0x1p-53, e = 4 * u * 3.5 * B;
  const double E = 2.02 * ((2 * e * sqrt(12 * thr) + 3 * e * e) * (1 + 3.01 * u) + 12.04 * u * thr);
  if (!(E < 0.5 * thr)) return __int_as_float(0x7f800000);
  return __double2float_ru(E);
}

__global__ void k_write_cells(const BNode* __restrict__ nodes, const int* __restrict__ leaf_parent,
                              const CellInfo* __restrict__ info, const unsigned* __restrict__ base,
                              const uint64_t* __restrict__ khi, const uint64_t* __restrict__ klo,
                              const double* __restrict__ nodes64, const int2* __restrict__ nodeids,
                              OvParams P, int n, Cell* cells, double* cell_lm, int2* cell_range,
                              int* lists, int* list_counts) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= 2 * n - 1) return;
  CellInfo ci = info[b];
  if (!ci.is_cell) return;
  int first, last, dX, parent;
  bnode_range(nodes, n, b, first, last, dX, parent, leaf_parent);
  int rank = 0;
  for (int p = parent; p >= 0 && nodes[p].first == first; p = nodes[p].parent)
    if (info[p].is_cell) ++rank;
  int idx = base[first] + rank;
  Cell c;
  memset(&c, 0, sizeof(c));
  c.skip = (int)base[last + 1];
  c.meta = ci.kind | (ci.ltop << 8) | (ci.lbot << 16);
  c.thr = DBL_MAX;
  double Lm = 0;
  if (ci.kind == CELL_LEAF1) {
    // the node's segment inline (segment_field, src/tangle.c:519-528)
    const double* nd = nodes64 + 6 * (size_t)first;
    int2 id = nodeids[first];
    c.a = id.x;
    c.b = id.y;
    for (int q = 0; q < 3; ++q) { c.x[q] = nd[q]; c.y[q] = nd[3 + q]; }
  } else if (ci.kind == CELL_LEAFN) {
    c.a = first;
    c.b = last - first + 1;
  }
  cell_range[idx] = make_int2(first, last - first + 1);
  if (ci.mac_level >= 0) {
    // replay the descent to the tested level to get the reference's box
    double lo[3] = {P.lo[0], P.lo[1], P.lo[2]}, hi[3] = {P.hi[0], P.hi[1], P.hi[2]};
    uint64_t h = khi[first], l = klo[first];
    for (int lev = 1; lev <= ci.mac_level; ++lev) {
      double cc[3], Lh[3], clo[3], chi[3];
      split_params(lo, hi, cc, Lh);
      child_box(lo, hi, cc, Lh, key_digit(h, l, lev), P.quadtree, clo, chi);
#pragma unroll
      for (int a = 0; a < 3; ++a) { lo[a] = clo[a]; hi[a] = chi[a]; }
    }
    Lm = box_max(lo, hi);
    c.thr = mac_threshold(Lm, P.theta);
    c.b = __float_as_int(mac_margin(P, c.thr));
    // moments are needed: file the cell by size for the moment kernels,
    // one atomic per class per warp (a list's order does not matter: each
    // cell's moments depend on its own nodes only)
    int count = last - first + 1;
    int cls = count <= 16 ? 0 : (count <= 4096 ? 1 : 2);
    const unsigned peers = __match_any_sync(__activemask(), cls);
    const int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
    int slot0 = 0;
    if (lane == leader) slot0 = atomicAdd(&list_counts[cls], __popc(peers));
    const int slot = __shfl_sync(peers, slot0, leader) + __popc(peers & ((1u << lane) - 1u));
    lists[cls * (size_t)(2 * n) + slot] = idx;
  }
  cells[idx] = c;
  cell_lm[idx] = Lm;
}

// ---------------------------------------------------------------- 5. nodes + moments
// per sorted node: r1, wrapped r2 (src/tangle.c:519-528) and ids for the skip rule
__global__ void k_nodes(OvParams P, const int* __restrict__ perm, const double* __restrict__ pos,
                        const int2* __restrict__ links, int n, double* nodes64, int2* nodeids) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int k = perm[i];
  int f = links[k].x;
  d3 a = ld3(pos, k);
  d3 b = f >= 0 ? pwrap(P, a, ld3(pos, f)) : a;
  double* o = nodes64 + 6 * (size_t)i;
  o[0] = a.x; o[1] = a.y; o[2] = a.z; o[3] = b.x; o[4] = b.y; o[5] = b.z;
  nodeids[i] = make_int2(k, f);
}

// Moments into the cell record: com, and kappa/4pi-scaled circulation and
// the four tensor entries the expansion reads, in FP64 and FP32.
__device__ __forceinline__ void write_moments(Cell* c, d3 com, d3 g, double m21, double m02,
                                              double m12, double m22, double f4pi) {
  double gs[3] = {g.x * f4pi, g.y * f4pi, g.z * f4pi};
  double ms[4] = {m21 * f4pi, m02 * f4pi, m12 * f4pi, m22 * f4pi};
  c->x[0] = com.x; c->x[1] = com.y; c->x[2] = com.z;
  for (int q = 0; q < 3; ++q) { c->y[q] = gs[q]; c->f_g[q] = (float)gs[q]; }
  for (int q = 0; q < 4; ++q) c->m[q] = ms[q];
  c->a = __float_as_int((float)ms[0]);
  c->f_m02 = (float)ms[1];
  c->f_m12 = (float)ms[2];
  c->f_m22 = (float)ms[3];
}

// Moments over a node range, one thread per cell (octree_update_means,
// src/octree.c:237-266): com = (sum of positions) * (1/N); gam = sum of the
// segment vectors; M = sum ds (x) (r - com).  Only the four entries of M the
// expansion reads are kept.
__global__ void k_moments_thread(const int* __restrict__ list, const int* __restrict__ list_count,
                                 Cell* cells, const int2* __restrict__ cell_range,
                                 const double* __restrict__ nodes64,
                                 const int2* __restrict__ nodeids, double f4pi) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= *list_count) return;
  int c = list[t];
  const int start = cell_range[c].x, count = cell_range[c].y;
  double sx = 0, sy = 0, sz = 0;
  for (int i = start; i < start + count; ++i) {
    const double* p = nodes64 + 6 * (size_t)i;
    sx += p[0]; sy += p[1]; sz += p[2];
  }
  double inv = 1.0 / count;
  d3 com = mk3(sx * inv, sy * inv, sz * inv);
  d3 g = mk3(0, 0, 0);
  double m21 = 0, m02 = 0, m12 = 0, m22 = 0;
  for (int i = start; i < start + count; ++i) {
    if (nodeids[i].y < 0) continue;
    const double* p = nodes64 + 6 * (size_t)i;
    d3 ds = mk3(p[3] - p[0], p[4] - p[1], p[5] - p[2]);
    d3 loc = mk3(p[0] - com.x, p[1] - com.y, p[2] - com.z);
    g = g + ds;
    m21 += ds.z * loc.y; m02 += ds.x * loc.z; m12 += ds.y * loc.z; m22 += ds.z * loc.z;
  }
  write_moments(cells + c, com, g, m21, m02, m12, m22, f4pi);
}

// same, one warp per cell (17..4096 nodes): lane-strided sums, then a
// butterfly over the warp
__device__ void moments_warp(int c, Cell* cells, const int2* __restrict__ cell_range,
                             const double* __restrict__ nodes64,
                             const int2* __restrict__ nodeids, double f4pi) {
  const int tid = threadIdx.x & 31;
  const int start = cell_range[c].x, count = cell_range[c].y;
  double s[3] = {0, 0, 0};
  for (int i = start + tid; i < start + count; i += 32) {
    const double* p = nodes64 + 6 * (size_t)i;
    s[0] += p[0]; s[1] += p[1]; s[2] += p[2];
  }
  for (int q = 0; q < 3; ++q) {
    double v = s[q];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    s[q] = v;
  }
  double inv = 1.0 / count;
  d3 com = mk3(s[0] * inv, s[1] * inv, s[2] * inv);
  double a[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int i = start + tid; i < start + count; i += 32) {
    if (nodeids[i].y < 0) continue;
    const double* p = nodes64 + 6 * (size_t)i;
    double dx = p[3] - p[0], dy = p[4] - p[1], dz = p[5] - p[2];
    double ly = p[1] - com.y, lz = p[2] - com.z;
    a[0] += dx; a[1] += dy; a[2] += dz;
    a[3] += dz * ly; a[4] += dx * lz; a[5] += dy * lz; a[6] += dz * lz;
  }
  for (int q = 0; q < 7; ++q) {
    double v = a[q];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    a[q] = v;
  }
  if (tid == 0) write_moments(cells + c, com, mk3(a[0], a[1], a[2]), a[3], a[4], a[5], a[6], f4pi);
}

__global__ void k_moments_warp(const int* __restrict__ list, const int* __restrict__ list_count,
                               Cell* cells, const int2* __restrict__ cell_range,
                               const double* __restrict__ nodes64,
                               const int2* __restrict__ nodeids, double f4pi) {
  int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= *list_count) return;
  moments_warp(list[w], cells, cell_range, nodes64, nodeids, f4pi);
}

// Cells of more than 4096 nodes: each cell's node range is cut into chunks of
// `chunk` nodes, one block of kMomThreads per (cell, chunk), so the largest
// cells (the root holds every node) spread over the GPU.  Partial sums per
// chunk land in part[(j * max_chunks + k) * 10 + ...] (3 position sums, then
// the 7 moment sums) and are added in chunk order, so the result does not
// depend on scheduling.
constexpr int kMomThreads = 256;
constexpr int kMomChunk = 8192;      // smallest chunk
constexpr int kMomMaxChunks = 64;    // chunks per cell at most

// sum of v over the block's threads, in a fixed order; valid in thread 0
template <int kN>
__device__ __forceinline__ void block_sum(double (&v)[kN], double* sh) {
  const int w = threadIdx.x >> 5, ln = threadIdx.x & 31;
#pragma unroll
  for (int q = 0; q < kN; ++q) {
    double x = v[q];
    for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
    v[q] = x;
  }
  if (ln == 0)
    for (int q = 0; q < kN; ++q) sh[w * kN + q] = v[q];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 0; q < kN; ++q) {
      double x = 0;
      for (int ww = 0; ww < kMomThreads / 32; ++ww) x += sh[ww * kN + q];
      v[q] = x;
    }
  }
}

// centre of mass of list cell j from its chunk position sums
__device__ __forceinline__ d3 chunked_com(const double* __restrict__ part, int j, int max_chunks,
                                          int count, int chunk) {
  const int nch = (count + chunk - 1) / chunk;
  double s[3] = {0, 0, 0};
  for (int k = 0; k < nch; ++k) {
    const double* pk = part + ((size_t)j * max_chunks + k) * 10;
    s[0] += pk[0]; s[1] += pk[1]; s[2] += pk[2];
  }
  const double inv = 1.0 / count;
  return mk3(s[0] * inv, s[1] * inv, s[2] * inv);
}

__global__ void __launch_bounds__(kMomThreads) k_moments_chunk_pos(
    const int* __restrict__ list, const int2* __restrict__ cell_range,
    const double* __restrict__ nodes64, int chunk, int max_chunks, double* part) {
  __shared__ double sh[(kMomThreads / 32) * 3];
  const int j = blockIdx.x, k = blockIdx.y;
  const int2 rg = cell_range[list[j]];
  const int lo = k * chunk;
  if (lo >= rg.y) return;
  const int hi = min(rg.y, lo + chunk);
  double s[3] = {0, 0, 0};
  for (int i = rg.x + lo + threadIdx.x; i < rg.x + hi; i += kMomThreads) {
    const double* p = nodes64 + 6 * (size_t)i;
    s[0] += p[0]; s[1] += p[1]; s[2] += p[2];
  }
  block_sum<3>(s, sh);
  if (threadIdx.x == 0) {
    double* o = part + ((size_t)j * max_chunks + k) * 10;
    o[0] = s[0]; o[1] = s[1]; o[2] = s[2];
  }
}

__global__ void __launch_bounds__(kMomThreads) k_moments_chunk_acc(
    const int* __restrict__ list, const int2* __restrict__ cell_range,
    const double* __restrict__ nodes64, const int2* __restrict__ nodeids, int chunk,
    int max_chunks, double* part) {
  __shared__ double sh[(kMomThreads / 32) * 7];
  __shared__ double sh_com[3];
  const int j = blockIdx.x, k = blockIdx.y;
  const int2 rg = cell_range[list[j]];
  const int lo = k * chunk;
  if (lo >= rg.y) return;
  const int hi = min(rg.y, lo + chunk);
  if (threadIdx.x == 0) {
    const d3 c = chunked_com(part, j, max_chunks, rg.y, chunk);
    sh_com[0] = c.x; sh_com[1] = c.y; sh_com[2] = c.z;
  }
  __syncthreads();
  const double cy = sh_com[1], cz = sh_com[2];
  double a[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int i = rg.x + lo + threadIdx.x; i < rg.x + hi; i += kMomThreads) {
    if (nodeids[i].y < 0) continue;
    const double* p = nodes64 + 6 * (size_t)i;
    const double dx = p[3] - p[0], dy = p[4] - p[1], dz = p[5] - p[2];
    const double ly = p[1] - cy, lz = p[2] - cz;
    a[0] += dx; a[1] += dy; a[2] += dz;
    a[3] += dz * ly; a[4] += dx * lz; a[5] += dy * lz; a[6] += dz * lz;
  }
  block_sum<7>(a, sh);
  if (threadIdx.x == 0) {
    double* o = part + ((size_t)j * max_chunks + k) * 10 + 3;
    for (int q = 0; q < 7; ++q) o[q] = a[q];
  }
}

// one thread per list cell: chunk sums in chunk order into the cell record
__global__ void k_moments_chunk_write(const int* __restrict__ list, const int* __restrict__ list_count,
                                      Cell* cells, const int2* __restrict__ cell_range, int chunk,
                                      int max_chunks, const double* __restrict__ part, double f4pi) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= *list_count) return;
  const int c = list[j];
  const int count = cell_range[c].y;
  const d3 com = chunked_com(part, j, max_chunks, count, chunk);
  const int nch = (count + chunk - 1) / chunk;
  double a[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int k = 0; k < nch; ++k) {
    const double* pk = part + ((size_t)j * max_chunks + k) * 10 + 3;
    for (int q = 0; q < 7; ++q) a[q] += pk[q];
  }
  write_moments(cells + c, com, mk3(a[0], a[1], a[2]), a[3], a[4], a[5], a[6], f4pi);
}

// a tangle of one node: the root is that node's leaf
__global__ void k_single_cell(Cell* cells, double* cell_lm, int2* cell_range,
                              const double* __restrict__ nodes64, const int2* __restrict__ nodeids) {
  Cell c;
  memset(&c, 0, sizeof(c));
  c.a = nodeids[0].x;
  c.b = nodeids[0].y;
  c.skip = 1;
  c.meta = CELL_LEAF1;
  c.thr = DBL_MAX;
  for (int q = 0; q < 3; ++q) { c.x[q] = nodes64[q]; c.y[q] = nodes64[3 + q]; }
  cells[0] = c;
  cell_lm[0] = 0;
  cell_range[0] = make_int2(0, 1);
}

}  // namespace

// ---------------------------------------------------------------- host driver
void ov_tree_release(OvTree* t) {
  DevBuf* bufs[] = {&t->keys, &t->keys_alt, &t->vals, &t->vals_alt, &t->stop, &t->hist,
                    &t->perm, &t->bnode, &t->cstart_cnt, &t->cbase, &t->cell_of, &t->cells,
                    &t->cell_lm, &t->cell_range, &t->nodes64, &t->nodeids, &t->nodes32, &t->counters,
                    &t->scratch, &t->scan_part, &t->mom_part};
  for (DevBuf* b : bufs) b->release();
  t->n_nodes = t->n_cells = t->built = 0;
}

// exclusive scan of v[0..m) in place (block sums in `part`)
static bool scan_excl(unsigned* v, int m, DevBuf& part, cudaStream_t st) {
  if (m <= 0) return true;
  const int nb = (m + kScanThreads - 1) / kScanThreads;
  if (!part.reserve(sizeof(unsigned) * (size_t)nb)) return false;
  unsigned* sums = part.as<unsigned>();
  k_scan_sums<<<nb, kScanThreads, 0, st>>>(v, m, sums);
  OV_LAUNCHED();
  k_scan_top<<<1, kScanThreads, 0, st>>>(sums, nb);
  OV_LAUNCHED();
  k_scan_apply<<<nb, kScanThreads, 0, st>>>(v, m, sums);
  OV_LAUNCHED();
  return ov_cuda_ok(cudaGetLastError(), "scan");
}

// Stable LSD radix sort of n 64-bit keys with int values, 8 passes of 8
// bits (k_rs_hist, the three-launch scan, k_rs_scatter).  (kb, vb) are the
// alternate buffers; after the even number of passes the sorted keys and
// values are back in (ka, va).
bool ov_radix_sort_u64(uint64_t* ka, int* va, uint64_t* kb, int* vb, int n, DevBuf& hist, DevBuf& scan_part,
                       cudaStream_t st) {
  if (n <= 0) return true;
  const int nb = (n + kRsTile - 1) / kRsTile;
  if (!hist.reserve(sizeof(unsigned) * 256 * (size_t)nb)) return false;
  for (int pass = 0; pass < 8; ++pass) {
    const int shift = 8 * pass;
    k_rs_hist<<<nb, kRsThreads, 0, st>>>(ka, n, shift, hist.as<unsigned>(), nb);
    OV_LAUNCHED();
    if (!scan_excl(hist.as<unsigned>(), 256 * nb, scan_part, st)) return false;
    k_rs_scatter<<<nb, kRsThreads, 0, st>>>(ka, va, kb, vb, n, shift, hist.as<unsigned>(), nb);
    OV_LAUNCHED();
    OV_TRY_CUDA(cudaGetLastError());
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  return true;
}

bool ov_tree_build(ov_state_impl* s, const double* pos, OvTree* T) {
  const int n = s->n;
  cudaStream_t st = s->stream;
  T->P = s->P;
  T->theta = s->P.theta;
  T->built = 0;
  const int nb_rs = (n + kRsTile - 1) / kRsTile;
  // key/value double buffers + low words + termination codes
  if (!T->keys.reserve(sizeof(uint64_t) * 2 * (size_t)n) ||      // hi (slot order), lo (slot order)
      !T->keys_alt.reserve(sizeof(uint64_t) * 2 * (size_t)n) ||  // hi alt, lo sorted
      !T->vals.reserve(sizeof(int) * 2 * (size_t)n) ||           // vals, term (slot)
      !T->vals_alt.reserve(sizeof(int) * 2 * (size_t)n) ||       // vals alt, term (sorted)
      !T->hist.reserve(sizeof(unsigned) * 256 * (size_t)(nb_rs > 0 ? nb_rs : 1)) ||
      !T->counters.reserve(128))
    return false;
  uint64_t* khi = T->keys.as<uint64_t>();
  uint64_t* klo_slot = khi + n;
  uint64_t* khi_alt = T->keys_alt.as<uint64_t>();
  uint64_t* klo = khi_alt + n;
  int* vals = T->vals.as<int>();
  int* term_slot = vals + n;
  int* vals_alt = T->vals_alt.as<int>();
  int* term = vals_alt + n;
  int* ctr = T->counters.as<int>();
  OV_TRY_CUDA(cudaMemsetAsync(ctr, 0, sizeof(int) * 16, st));
  if (n > 0) {
    k_keys<<<(n + 255) / 256, 256, 0, st>>>(s->P, pos, s->status.as<int2>(), n, khi, klo_slot, vals,
                                             term_slot, ctr);
    OV_LAUNCHED();
    OV_TRY_CUDA(cudaGetLastError());
  }
  int hc[4] = {0, 0, 0, 0};
  OV_TRY_CUDA(cudaMemcpyAsync(hc, ctr, sizeof(hc), cudaMemcpyDeviceToHost, st));
  OV_TRY_CUDA(cudaStreamSynchronize(st));
  if (hc[1]) {
    ov_set_error(OV_ERR_TREE_DEPTH,
                 "octree: the box / BH_grain ratio needs more than %d levels", kMaxLevels);
    return false;
  }
  const int na = hc[0];
  T->n_nodes = na;
  // a node outside the root box takes digit 8 at level 1, so these nodes
  // sort after every node inside it: the last n_drop_root of the order
  T->n_drop_root = hc[3];
  // radix sort over the high word (8 passes of 8 bits), stable; vals_alt's
  // second half holds the sorted term codes, so the values alternate with a
  // separate scratch.  The sorted data ends back in khi / vals.
  uint64_t* ka = khi;
  int* va = vals;
  if (!T->scratch.reserve(sizeof(int) * (size_t)n + 16)) return false;
  if (!ov_radix_sort_u64(khi, vals, khi_alt, T->scratch.as<int>(), n, T->hist, T->scan_part, st)) return false;
  if (!T->perm.reserve(sizeof(int) * (size_t)(n > 0 ? n : 1))) return false;
  int* perm = T->perm.as<int>();
  if (n > 0) {
    OV_TRY_CUDA(cudaMemcpyAsync(perm, va, sizeof(int) * n, cudaMemcpyDeviceToDevice, st));
    k_gather_lo<<<(n + 255) / 256, 256, 0, st>>>(perm, klo_slot, term_slot, klo, term, n);
    OV_LAUNCHED();
    if (na > 0) {
      k_fix_ties<<<(na + 255) / 256, 256, 0, st>>>(ka, klo, perm, term, na);
      OV_LAUNCHED();
    }
    OV_TRY_CUDA(cudaGetLastError());
  }
  const uint64_t* hi_sorted = ka;
  // sorted node table for the walk
  if (!T->nodes64.reserve(sizeof(double) * 6 * (size_t)(na > 0 ? na : 1)) ||
      !T->nodeids.reserve(sizeof(int2) * (size_t)(na > 0 ? na : 1)))
    return false;
  if (na > 0) {
    k_nodes<<<(na + 255) / 256, 256, 0, st>>>(s->P, perm, pos, s->links.as<int2>(), na,
                                               T->nodes64.as<double>(), T->nodeids.as<int2>());
    OV_LAUNCHED();
    OV_TRY_CUDA(cudaGetLastError());
  }
  if (na == 0) {
    T->n_cells = 0;
    T->built = 1;
    return true;
  }
  // radix tree + cells
  const int nbin = 2 * na - 1;
  size_t bn_bytes = sizeof(BNode) * (size_t)(na > 1 ? na - 1 : 1) + sizeof(int) * (size_t)na;
  if (!T->bnode.reserve(bn_bytes) ||
      !T->cstart_cnt.reserve(sizeof(CellInfo) * (size_t)nbin) ||
      !T->cbase.reserve(sizeof(unsigned) * (size_t)(na + 1)) ||
      !T->cells.reserve(sizeof(Cell) * (size_t)nbin) ||
      !T->cell_lm.reserve(sizeof(double) * (size_t)nbin) ||
      !T->cell_range.reserve(sizeof(int2) * (size_t)nbin) ||
      !T->cell_of.reserve(sizeof(int) * (3 * 2 * (size_t)na) + 64))
    return false;
  BNode* bn = T->bnode.as<BNode>();
  int* leaf_parent = reinterpret_cast<int*>(reinterpret_cast<char*>(T->bnode.p) +
                                            sizeof(BNode) * (size_t)(na > 1 ? na - 1 : 1));
  CellInfo* info = T->cstart_cnt.as<CellInfo>();
  unsigned* base = T->cbase.as<unsigned>();
  int* lists = T->cell_of.as<int>();
  int* list_counts = ctr + 4;
  Cell* cells = T->cells.as<Cell>();
  double* cell_lm = T->cell_lm.as<double>();
  int2* cell_range = T->cell_range.as<int2>();
  if (na == 1) {
    k_single_cell<<<1, 1, 0, st>>>(cells, cell_lm, cell_range, T->nodes64.as<double>(),
                                   T->nodeids.as<int2>());
    OV_LAUNCHED();
    OV_TRY_CUDA(cudaGetLastError());
    T->n_cells = 1;
  } else {
    k_karras<<<(na - 1 + 255) / 256, 256, 0, st>>>(hi_sorted, klo, na, bn, leaf_parent);
    OV_LAUNCHED();
    OV_TRY_CUDA(cudaMemsetAsync(base, 0, sizeof(unsigned) * (na + 1), st));
    k_classify<<<(nbin + 255) / 256, 256, 0, st>>>(bn, leaf_parent, term, na, info, base);
    OV_LAUNCHED();
    if (!scan_excl(base, na + 1, T->scan_part, st)) return false;
    k_write_cells<<<(nbin + 255) / 256, 256, 0, st>>>(bn, leaf_parent, info, base, hi_sorted, klo,
                                                      T->nodes64.as<double>(), T->nodeids.as<int2>(),
                                                      s->P, na, cells, cell_lm, cell_range, lists,
                                                      list_counts);
    OV_LAUNCHED();
    OV_TRY_CUDA(cudaGetLastError());
    unsigned nc = 0;
    int lc[3] = {0, 0, 0};
    OV_TRY_CUDA(cudaMemcpyAsync(&nc, base + na, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    OV_TRY_CUDA(cudaMemcpyAsync(lc, list_counts, sizeof(lc), cudaMemcpyDeviceToHost, st));
    OV_TRY_CUDA(cudaStreamSynchronize(st));
    T->n_cells = (int)nc;
    const double f4 = s->P.f4pi;
    if (lc[0] > 0) {
      k_moments_thread<<<(lc[0] + 127) / 128, 128, 0, st>>>(lists, list_counts, cells, cell_range,
                                                            T->nodes64.as<double>(), T->nodeids.as<int2>(), f4);
      OV_LAUNCHED();
    }
    if (lc[1] > 0) {
      k_moments_warp<<<(lc[1] * 32 + 255) / 256, 256, 0, st>>>(lists + 2 * (size_t)na, list_counts + 1,
                                                              cells, cell_range, T->nodes64.as<double>(),
                                                              T->nodeids.as<int2>(), f4);
      OV_LAUNCHED();
    }
    if (lc[2] > 0) {
      // chunks of at least kMomChunk nodes, at most kMomMaxChunks per cell
      const int chunk = std::max(kMomChunk, (na + kMomMaxChunks - 1) / kMomMaxChunks);
      const int max_chunks = (na + chunk - 1) / chunk;
      if (!T->mom_part.reserve(sizeof(double) * 10 * (size_t)lc[2] * max_chunks)) return false;
      const int* blist = lists + 4 * (size_t)na;
      double* part = T->mom_part.as<double>();
      const dim3 grid(lc[2], max_chunks);
      k_moments_chunk_pos<<<grid, kMomThreads, 0, st>>>(blist, cell_range, T->nodes64.as<double>(), chunk,
                                                         max_chunks, part);
      OV_LAUNCHED();
      k_moments_chunk_acc<<<grid, kMomThreads, 0, st>>>(blist, cell_range, T->nodes64.as<double>(),
                                                         T->nodeids.as<int2>(), chunk, max_chunks, part);
      OV_LAUNCHED();
      k_moments_chunk_write<<<(lc[2] + 127) / 128, 128, 0, st>>>(blist, list_counts + 2, cells, cell_range,
                                                                  chunk, max_chunks, part, f4);
      OV_LAUNCHED();
    }
    OV_TRY_CUDA(cudaGetLastError());
  }
  OvStatsAcc& acc = ov_stats_tls();
  acc.cells = T->n_cells;
  T->built = 1;
  return true;
}
