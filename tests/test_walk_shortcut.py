"""The multi-image walk's shortcut decisions, restated on the CPU.

For each cell the walk computes the target's own wrapped squared distance q0
with the reference's FP64 operations (octree_get_vs, src/octree.c:284-296).
When q0 >= thr + E it takes every image's opening test as passed; when
q0 < thr - E and no axis of the unwrapped difference c - r reaches hw it takes
every image's test as failed.  E is the cell's margin (ov_tree.cu,
mac_margin) and hw the per-axis limit (ov_walk.cu, ImageShortcut).  This
test restates both from their derivation and checks, on targets and centres
of mass placed near the threshold, that every one of the 27 images decides
as the shortcut says when each image is tested with the reference's own
operations.  Python floats are IEEE doubles with round-to-nearest, like the
kernel's __dadd_rn / __dsub_rn / __dmul_rn.
"""
import math
import random

import numpy as np

U = 2.0 ** -53


def wrapped_sq(v, c, L, periodic):
    cc = c
    if periodic:
        d = c - v
        if d > L * 0.5:
            cc = c - L
        elif d < -L * 0.5:
            cc = c + L
    u = v - cc
    return u * u


def img_coord(r, L, i):
    return r if i == 1 else (r - (-L) if i == 0 else r - L)


def margin(lo, hi, thr):
    """mac_margin: FP32 rounded up, infinity when above thr / 2."""
    B = max(abs(a) + abs(b) for a, b in zip(lo, hi))
    e = 4 * U * 3.5 * B
    E = 2.02 * ((2 * e * math.sqrt(12 * thr) + 3 * e * e) * (1 + 3.01 * U) + 12.04 * U * thr)
    if not E < 0.5 * thr:
        return math.inf
    f = np.float32(E)
    if float(f) < E:
        f = np.nextafter(f, np.float32(np.inf))
    return float(f)


def half_width(lo, hi):
    B = max(abs(a) + abs(b) for a, b in zip(lo, hi))
    return [0.5 * (h - l) - 8 * U * 3.5 * B for l, h in zip(lo, hi)]


def image_q(r, c, L, i3):
    return (wrapped_sq(img_coord(r[0], L[0], i3[0]), c[0], L[0], True)
            + wrapped_sq(img_coord(r[1], L[1], i3[1]), c[1], L[1], True)) \
        + wrapped_sq(img_coord(r[2], L[2], i3[2]), c[2], L[2], True)


def test_shortcut_decisions_match_every_image():
    rng = random.Random(20240611)
    checked = {"pass": 0, "fail": 0}
    for trial in range(20000):
        off = rng.choice([0.0, -0.5, 3.0, -17.25])
        size = rng.choice([0.1, 1.0, 2 * math.pi, 7.0])
        lo = [off * size] * 3
        hi = [lo[a] + size * rng.uniform(0.8, 1.2) for a in range(3)]
        L = [hi[a] - lo[a] for a in range(3)]
        # a cell centre of mass inside the box, a target within a quarter box
        c = [rng.uniform(lo[a], hi[a]) for a in range(3)]
        # cell sizes from half the box down to 1e-9 of it
        side = size * 10.0 ** rng.uniform(-9, -0.3)
        thr = (side / 0.5) ** 2
        # target at a distance near sqrt(thr), within a few ulps to 1e-6 of it
        direction = [rng.gauss(0, 1) for _ in range(3)]
        nrm = math.sqrt(sum(x * x for x in direction))
        rel = rng.choice([1.0, -1.0]) * 10.0 ** rng.uniform(-16, -6)
        dist = math.sqrt(thr) * (1 + rel)
        r = [c[a] + direction[a] / nrm * dist for a in range(3)]
        mode = rng.random()
        if mode < 0.3:
            # across a periodic boundary: the target sits near the other face
            ax = rng.randrange(3)
            r[ax] += L[ax] if r[ax] < 0.5 * (lo[ax] + hi[ax]) else -L[ax]
        elif mode < 0.6:
            # about half a box from the centre of mass along one axis (where
            # one image per axis stops matching the target), the threshold
            # within 1e-12 .. 1e-6 of the target's distance
            ax = rng.randrange(3)
            c[ax] = rng.uniform(lo[ax], hi[ax])
            half = 0.5 * L[ax] * (1 + rng.uniform(-1e-6, 1e-6))
            r[ax] = c[ax] - half if rng.random() < 0.5 else c[ax] + half
            q_t = (wrapped_sq(r[0], c[0], L[0], True) + wrapped_sq(r[1], c[1], L[1], True)) \
                + wrapped_sq(r[2], c[2], L[2], True)
            thr = q_t * (1 + rng.choice([1.0, -1.0]) * 10.0 ** rng.uniform(-12, -6))
        if any(not (lo[a] - 0.25 * L[a] <= r[a] <= hi[a] + 0.25 * L[a]) for a in range(3)):
            continue
        E = margin(lo, hi, thr)
        hw = half_width(lo, hi)
        d = [c[a] - r[a] for a in range(3)]
        q0 = (wrapped_sq(r[0], c[0], L[0], True) + wrapped_sq(r[1], c[1], L[1], True)) \
            + wrapped_sq(r[2], c[2], L[2], True)
        if q0 >= thr + E:
            kind = "pass"
        elif q0 < thr - E and all(abs(d[a]) <= hw[a] for a in range(3)):
            kind = "fail"
        else:
            continue
        checked[kind] += 1
        for ix in range(3):
            for iy in range(3):
                for iz in range(3):
                    q = image_q(r, c, L, (ix, iy, iz))
                    assert (q >= thr) == (kind == "pass"), (trial, kind, ix, iy, iz, q, thr, E)
    # both shortcuts were exercised, many times each
    assert checked["pass"] > 2000 and checked["fail"] > 2000, checked


def test_margin_scales_with_rounding():
    # a margin well below the cell's own threshold for ordinary cells, and
    # infinity (no shortcut) only when the cell is near the box's rounding
    lo, hi = [0.0] * 3, [1.0] * 3
    assert margin(lo, hi, 1e-6) < 1e-13 * 1.0
    assert margin(lo, hi, (1e-3 / 0.5) ** 2) / (1e-3 / 0.5) ** 2 < 1e-10
    assert margin(lo, hi, 1e-58) == math.inf
