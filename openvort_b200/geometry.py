"""Seeded tangle generators for the benchmark and test workloads.

Rings are placed with the reference's circle geometry (add_circle,
src/vortex_utils.c:52-99), so the CPU reference and the GPU receive identical
positions and links.  All randomness comes from numpy's default_rng(seed).
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np

from .tangle import EMPTY, FREE, HostTangle, ring_points


def rings_to_tangle(rings: Sequence[np.ndarray], box_lo, box_hi, boundary: str,
                    wrap: bool = False, empty_slots: int = 0, alloc=np.empty) -> HostTangle:
    """Concatenate closed loops (each an (n, 3) array in order) into one
    tangle: node i of a loop links forward to i+1 and back to i-1."""
    pos, fwd, rev = [], [], []
    off = 0
    for r in rings:
        n = len(r)
        idx = np.arange(n)
        pos.append(r)
        fwd.append(off + (idx + 1) % n)
        rev.append(off + (idx - 1) % n)
        off += n
    pos = np.concatenate(pos) if pos else np.zeros((0, 3))
    fwd = np.concatenate(fwd).astype(np.int32) if fwd else np.zeros(0, np.int32)
    rev = np.concatenate(rev).astype(np.int32) if rev else np.zeros(0, np.int32)
    status = np.full(len(pos), FREE, np.int32)
    if wrap:
        lo = np.asarray(box_lo, dtype=np.float64)
        L = np.asarray(box_hi, dtype=np.float64) - lo
        pos = lo + np.mod(pos - lo, L)
    if empty_slots:
        # EMPTY holes interleaved with the nodes, as remeshing leaves them
        n = len(pos)
        total = n + empty_slots
        rng = np.random.default_rng(12345)
        holes = np.sort(rng.choice(total, size=empty_slots, replace=False))
        keep = np.setdiff1d(np.arange(total), holes)
        newpos = np.zeros((total, 3))
        newpos[keep] = pos
        newpos[holes] = 0.5 * (np.asarray(box_lo) + np.asarray(box_hi))
        remap = np.full(n, -1, np.int64)
        remap[np.arange(n)] = keep
        nf = np.full(total, -1, np.int32)
        nr = np.full(total, -1, np.int32)
        nf[keep] = remap[fwd]
        nr[keep] = remap[rev]
        st = np.full(total, EMPTY, np.int32)
        st[keep] = FREE
        pos, fwd, rev, status = newpos, nf, nr, st
    return HostTangle(pos, fwd, rev, status, None, box_lo, box_hi, boundary, alloc=alloc)


def single_ring(n: int = 256, radius: float = 1e-2, center=(0.0, 0.0, 0.0),
                direction=(0.0, 0.0, 1.0), box_half: float = 0.05, alloc=np.empty) -> HostTangle:
    """One circular ring in open space; the box encloses it (the box only
    matters to the Barnes-Hut tree, src/tangle.c:102-105)."""
    c = np.asarray(center, dtype=np.float64)
    r = ring_points(c, direction, radius, n)
    return rings_to_tangle([r], c - box_half, c + box_half, "open", alloc=alloc)


def random_ring_tangle(seed: int, n_rings: int, D: float, r_frac=(0.02, 0.05), dl=None,
                       boundary: str = "periodic-26", empty_slots: int = 0,
                       alloc=np.empty) -> HostTangle:
    """Rings with centres uniform in [0, D]^3, normals uniform on the sphere,
    radii uniform in [r_frac] * D, about 2 pi r / dl points each; positions
    wrapped into the periodic box."""
    rng = np.random.default_rng(seed)
    dl = D / 200 if dl is None else dl
    rings = []
    for _ in range(n_rings):
        c = rng.uniform(0.0, D, size=3)
        d = rng.normal(size=3)
        d /= np.sqrt(d @ d)
        r = rng.uniform(r_frac[0] * D, r_frac[1] * D)
        n = max(5, int(round(2 * np.pi * r / dl)))
        rings.append(ring_points(c, d, r, n))
    return rings_to_tangle(rings, (0.0, 0.0, 0.0), (D, D, D), boundary, wrap=True,
                           empty_slots=empty_slots, alloc=alloc)


def rings_for_points(target_points: int, D: float, r_frac=(0.02, 0.05), dl=None) -> int:
    """Number of rings whose expected point count is target_points."""
    dl = D / 200 if dl is None else dl
    mean_n = 2 * np.pi * 0.5 * (r_frac[0] + r_frac[1]) * D / dl
    return max(1, int(round(target_points / mean_n)))


def ring_pair_system(rng: np.random.Generator, kind: str, n_total: int,
                     r_range=(5e-3, 2e-2)) -> List[np.ndarray]:
    """Two rings on the z axis: 'leapfrog' (same direction) or 'headon'
    (opposite directions), radii uniform in r_range, points split by length."""
    r1, r2 = rng.uniform(*r_range, size=2)
    n1 = max(8, int(round(n_total * r1 / (r1 + r2))))
    n2 = max(8, n_total - n1)
    gap = 0.5 * (r1 + r2)
    if kind == "leapfrog":
        a = ring_points((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), r1, n1)
        b = ring_points((0.0, 0.0, gap), (0.0, 0.0, 1.0), r2, n2)
    else:
        a = ring_points((0.0, 0.0, -gap), (0.0, 0.0, 1.0), r1, n1)
        b = ring_points((0.0, 0.0, gap), (0.0, 0.0, -1.0), r2, n2)
    return [a, b]


def ring_pair_ensemble(seed: int, n_systems: int, n_range=(64, 2048), r_range=(5e-3, 2e-2),
                       alloc=np.empty) -> Tuple[HostTangle, np.ndarray, List[List[np.ndarray]]]:
    """Independent open-boundary systems for the batched path: each a coaxial
    ring pair, leapfrogging or head-on (chosen at random), radii uniform in
    r_range, total points uniform in n_range.  Returns the concatenated
    tangle, the n_systems + 1 slot offsets, and each system's rings."""
    rng = np.random.default_rng(seed)
    systems = []
    for _ in range(n_systems):
        kind = "leapfrog" if rng.uniform() < 0.5 else "headon"
        n_total = int(rng.integers(n_range[0], n_range[1] + 1))
        systems.append(ring_pair_system(rng, kind, n_total, r_range))
    rings = [r for sys_ in systems for r in sys_]
    half = 2.0 * r_range[1] + 0.05
    t = rings_to_tangle(rings, (-half,) * 3, (half,) * 3, "open", alloc=alloc)
    sizes = [sum(len(r) for r in sys_) for sys_ in systems]
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    return t, offsets, systems


def kelvin_ring(seed: int, n: int = 4096, radius: float = 1e-2, modes=(2, 32),
                sigma: float = 1e-4) -> np.ndarray:
    """A ring with a seeded Kelvin-wave perturbation: radial and axial
    displacements sum_m a_m cos(m phi + phase_m), amplitudes N(0, sigma^2)."""
    rng = np.random.default_rng(seed)
    base = ring_points((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), radius, n)
    phi = 2 * np.pi * np.arange(n) / n
    dr = np.zeros(n)
    dz = np.zeros(n)
    for m in range(modes[0], modes[1] + 1):
        a, b = rng.normal(0.0, sigma, size=2)
        p1, p2 = rng.uniform(0, 2 * np.pi, size=2)
        dr += a * np.cos(m * phi + p1)
        dz += b * np.cos(m * phi + p2)
    rad = base[:, :2] / np.linalg.norm(base[:, :2], axis=1)[:, None]
    out = base.copy()
    out[:, :2] += rad * dr[:, None]
    out[:, 2] += dz
    return out


def wall_half_ring(n: int = 64, radius: float = 1e-2, box=0.05) -> HostTangle:
    """A half ring standing on the z = 0 mirror wall with both ends pinned
    (pinned one-sided stencils, mirror image, boundary velocity)."""
    phi = np.linspace(0.0, np.pi, n)
    pos = np.stack([radius * np.cos(phi), np.zeros(n), radius * np.sin(phi)], axis=1)
    pos[0, 2] = 0.0
    pos[-1, 2] = 0.0
    idx = np.arange(n)
    fwd = np.where(idx < n - 1, idx + 1, -1).astype(np.int32)
    rev = np.where(idx > 0, idx - 1, -1).astype(np.int32)
    status = np.full(n, FREE, np.int32)
    status[0] = status[-1] = 1  # PINNED
    pin = np.full(n, -1, np.int32)
    pin[0] = pin[-1] = 4        # Z_L
    return HostTangle(pos, fwd, rev, status, pin, (-box, -box, 0.0), (box, box, 2 * box),
                      "wall-1-open")


def perturb_spacing(t: HostTangle, seed: int, frac_move: float = 0.05, n_gaps: int = 6) -> HostTangle:
    """Uneven resolution for remesh workloads, in place: a fraction of the
    free nodes pushed 30-80% of the way to their forward neighbour (a short
    segment and a long one), and n_gaps pairs of consecutive free nodes taken
    out, their neighbours linked across the gap (one segment three spacings
    long)."""
    rng = np.random.default_rng(seed)
    act = np.nonzero(t.active)[0]
    free = act[t.stat[act, 0] == FREE]
    periodic = t.boundary.startswith("periodic")
    L = np.asarray(t.box_hi, dtype=np.float64) - np.asarray(t.box_lo, dtype=np.float64)
    for k in rng.choice(free, size=max(1, int(frac_move * len(free))), replace=False):
        f = t.links[k, 0]
        if f < 0:
            continue
        d = t.pos[f] - t.pos[k]
        if periodic:
            d = d - L * np.round(d / L)
        t.pos[k] += rng.uniform(0.3, 0.8) * d
    done = set()
    gaps = 0
    for k in rng.choice(free, size=min(len(free), 4 * n_gaps), replace=False):
        if gaps >= n_gaps:
            break
        a = int(k)
        b = int(t.links[a, 0])
        if b < 0 or t.stat[b, 0] != FREE:
            continue
        p, nx = int(t.links[a, 1]), int(t.links[b, 0])
        if p < 0 or nx < 0 or nx == p or len({p, a, b, nx} & done):
            continue
        t.links[p, 0], t.links[nx, 1] = nx, p
        for q in (a, b):
            t.links[q] = -1
            t.stat[q, 0] = EMPTY
        done |= {p, a, b, nx}
        gaps += 1
    return t


def relabel_slots(t: HostTangle, seed: int) -> HostTangle:
    """The same tangle with its slots in a seeded random order (links
    renumbered; vels, tangents, normals and dxi carried along)."""
    rng = np.random.default_rng(seed)
    n = len(t.pos)
    perm = rng.permutation(n)               # old slot k -> new slot perm[k]
    inv = np.empty(n, np.int64)
    inv[perm] = np.arange(n)

    def renum(x):
        return np.where(x >= 0, perm[np.maximum(x, 0)], -1).astype(np.int32)

    out = HostTangle(t.pos[inv], renum(t.links[inv, 0]), renum(t.links[inv, 1]), t.stat[inv, 0],
                     t.stat[inv, 1], t.box_lo, t.box_hi, t.boundary)
    for name in ("vels", "tangents", "normals", "dxi"):
        getattr(out, name)[:] = getattr(t, name)[inv]
    return out


def join_tangles(parts: Sequence[HostTangle], box_lo, box_hi, boundary: str) -> HostTangle:
    """Several tangles' slots side by side in one tangle."""
    pos, fwd, rev, st, pin = [], [], [], [], []
    off = 0
    for t in parts:
        n = len(t.pos)
        pos.append(t.pos)
        fwd.append(np.where(t.links[:, 0] >= 0, t.links[:, 0] + off, -1))
        rev.append(np.where(t.links[:, 1] >= 0, t.links[:, 1] + off, -1))
        st.append(t.stat[:, 0])
        pin.append(t.stat[:, 1])
        off += n
    cat = np.concatenate
    return HostTangle(cat(pos), cat(fwd).astype(np.int32), cat(rev).astype(np.int32), cat(st).astype(np.int32),
                      cat(pin).astype(np.int32), box_lo, box_hi, boundary)
