// ov_links.cuh - walks along the vortex links on the device: the
// position a few links away (step_node, src/tangle.c:165-200) and the arc
// length along the stored segment lengths (arc_length, src/tangle.c:208-243),
// both reflecting at pinned ends as the reference does.
#pragma once

#include "ov_internal.h"

namespace {

struct Links {
  const int2* lk;   // (forward, reverse) per slot
  const int2* st;   // (status, pin_wall) per slot
};

__device__ __forceinline__ bool pinned_any(int st) { return st == OV_PINNED || st == OV_PINNED_SLIP; }

// Position `where` links away from node i (step_node, src/tangle.c:165-200).
// Walking off a pinned end continues backwards on the mirror image of the
// vortex.  Returns false on a broken link.
__device__ bool step_node(const OvParams& P, const Links& L, const double* pos, int i,
                          int where, d3& out) {
  int faces[8];
  int nf = 0;
  int cur = i, w = where;
  for (int it = 0; it < 16 && w != 0; ++it) {
    int2 st = L.st[cur];
    bool pin = pinned_any(st.x);
    int2 lk = L.lk[cur];
    int nx = w > 0 ? lk.x : lk.y;
    if (nx >= 0) {
      cur = nx;
      w += w > 0 ? -1 : 1;
    } else if (pin && nf < 8) {
      faces[nf++] = st.y;
      w = -w;
    } else {
      return false;
    }
  }
  if (w != 0) return false;
  d3 p = ld3(pos, cur);
  for (int f = nf - 1; f >= 0; --f) {
    int face = faces[f];
    int c = face >> 1;
    double wp = (face & 1) ? P.hi[c] : P.lo[c];
    set_axis(p, c, 2.0 * wp - axis_of(p, c));
  }
  out = p;
  return true;
}

// Arc length `dist` links away along the stored segment lengths
// (arc_length, src/tangle.c:208-243); reverses at a pinned end.
__device__ bool arc_length(const Links& L, const double* dxi, int k, int dist, double& out) {
  double acc = 0;
  int cur = k, d = dist;
  for (int it = 0; it < 16 && d != 0; ++it) {
    bool pin = pinned_any(L.st[cur].x);
    int2 lk = L.lk[cur];
    if (d > 0) {
      if (lk.x < 0) {
        if (!pin) return false;
        d = -d;
        continue;
      }
      acc += dxi[cur];
      cur = lk.x;
      --d;
    } else {
      if (lk.y < 0) {
        if (!pin) return false;
        d = -d;
        continue;
      }
      acc += dxi[lk.y];
      cur = lk.y;
      ++d;
    }
  }
  if (d != 0) return false;
  out = acc;
  return true;
}

}  // namespace
