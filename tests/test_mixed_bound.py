"""The error bound of the mixed reconnection sums, restated on the CPU.

k_direct_mixed_points (ov_direct.cu) evaluates far segment-target pairs in
FP32 and gives each target E = 256u kappa/4pi sum |d| / |R|^2 (u = 2^-24)
over those pairs, as a bound on |mixed - FP64| of its sum.  The kernel's
comment splits the budget: input rounding and formula evaluation <= 53u per
unit of kappa/4pi |d| / |R|^2 for each pair, and the FP32 partial sums of 16
terms <= 26u of the same sum.  This test emulates the kernel's FP32
arithmetic with numpy (each float32 operation rounds once; fused multiply-
adds are formed in float64 and rounded once), with the hardware reciprocal
square root and reciprocal perturbed by their documented relative errors
(2^-22.9 and one ulp) in random directions, on pairs spread over a box at
distances from 4 to 4000 segment lengths, including pairs just outside the
reference's colinearity cut-off (src/tangle.c:505-506).  It checks each
pair against 64u and every 16-term partial sum against the whole 256u.
"""
import numpy as np

U = 2.0 ** -24
F32 = np.float32
F4PI = 9.97e-4 / (4 * np.pi)


def f32(x):
    return np.asarray(x, dtype=np.float64).astype(F32)


def fma32(a, b, c):
    """a * b + c rounded once to float32 (the product of two floats is exact in float64)"""
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(F32)


def two_float(x):
    hi = f32(x)
    lo = f32(x - hi.astype(np.float64))
    return hi, lo


def seg64(r1, r2, t):
    """the reference's segment formula in FP64 (segment_field1, src/tangle.c:486-514)"""
    R, Rp = r1 - t, r2 - t
    a, b = np.linalg.norm(R, axis=-1), np.linalg.norm(Rp, axis=-1)
    RRp = np.sum(R * Rp, axis=-1)
    s = F4PI * (a + b) / (a * b * (a * b + RRp))
    return np.cross(R, Rp) * s[..., None]


def pair32(r1, r2, t, rng):
    """one pair as pair_interact evaluates it (two-float offsets from the
    origin), without the kappa/4pi factor; returns (C s, 1 - cos)"""
    ahi, alo = two_float(r1)
    thi, tlo = two_float(t)
    R = (ahi - thi) + (alo - tlo)           # float32 ops
    d = f32(r2 - r1)
    Rx, Ry, Rz = R[..., 0], R[..., 1], R[..., 2]
    dx, dy, dz = d[..., 0], d[..., 1], d[..., 2]
    d2 = fma32(dx, dx, fma32(dy, dy, dz * dz))
    R2 = fma32(Rz, Rz, fma32(Ry, Ry, Rx * Rx))
    Rd = fma32(Rz, dz, fma32(Ry, dy, Rx * dx))
    Q2 = fma32(F32(2.0) * np.ones_like(Rd), Rd, R2 + d2)
    n = R2.shape

    def approx(x, rel):
        return (x.astype(np.float64) * (1.0 + rel * rng.choice([-1.0, 1.0], size=n))).astype(F32)
    ia = approx(1.0 / np.sqrt(R2.astype(np.float64)), 2.0 ** -22.9)
    ib = approx(1.0 / np.sqrt(Q2.astype(np.float64)), 2.0 ** -22.9)
    u = ia * ib
    den = fma32(R2 + Rd, u, F32(1.0) * np.ones_like(u))
    r = approx(1.0 / den.astype(np.float64), 2.0 ** -23)
    w = u * r
    s = (ia + ib) * w
    Cx = fma32(Ry, dz, Rz * (-dy))
    Cy = fma32(Rz, dx, Rx * (-dz))
    Cz = fma32(Rx, dy, Ry * (-dx))
    tc = fma32(Cz, Cz, fma32(Cy, Cy, Cx * Cx)) * (u * w)
    return np.stack([Cx, Cy, Cz], axis=-1), s, tc


def far_pairs(rng, n, colinear=False):
    """targets anywhere in [-0.5, 0.5]^3, segments of 1e-4 .. 1e-3 cm at
    4 .. 4000 lengths from them"""
    t = rng.uniform(-0.5, 0.5, size=(n, 3))
    ln = 10 ** rng.uniform(-4, -3, size=n)
    dist = ln * 10 ** rng.uniform(np.log10(4.5), np.log10(4000), size=n)
    e = rng.normal(size=(n, 3))
    e /= np.linalg.norm(e, axis=1)[:, None]
    r1 = t + e * dist[:, None]
    dirn = rng.normal(size=(n, 3))
    if colinear:
        # segment nearly along the line of sight: 1 - cos just above 1e-8
        perp = dirn - np.sum(dirn * e, axis=1)[:, None] * e
        perp /= np.linalg.norm(perp, axis=1)[:, None]
        ang = (dist / ln) * np.sqrt(2e-8) * rng.uniform(1.05, 3.0, size=n)
        dirn = e + perp * ang[:, None]
    dirn /= np.linalg.norm(dirn, axis=1)[:, None]
    r2 = r1 + dirn * ln[:, None]
    return r1, r2, t


def per_pair_check(rng, colinear):
    r1, r2, t = far_pairs(rng, 200_000, colinear)
    C, s, tc = pair32(r1, r2, t, rng)
    ok = tc > F32(1e-8 * (1 + 2.5e-3))                   # the pairs the kernel keeps in FP32
    v32 = F4PI * (C.astype(np.float64) * s.astype(np.float64)[:, None])
    v64 = seg64(r1, r2, t)
    unit = F4PI * np.linalg.norm(r2 - r1, axis=1) / np.sum((r1 - t) ** 2, axis=1)
    err = np.linalg.norm(v32 - v64, axis=1)
    return ok, err / unit, (v32, v64, unit)


def test_each_far_pair_within_its_share_of_the_bound():
    rng = np.random.default_rng(11)
    for colinear in (False, True):
        ok, ratio, _ = per_pair_check(rng, colinear)
        assert ok.sum() > 1000
        worst = ratio[ok].max()
        assert worst < 64 * U, (colinear, worst / U)


def test_partial_sums_within_the_whole_bound():
    """16 pairs per FP32 partial sum, as the kernel flushes them, against the
    FP64 sum of the FP64 formula: within 256u of sum kappa/4pi |d| / |R|^2."""
    rng = np.random.default_rng(12)
    r1, r2, t0 = far_pairs(rng, 16 * 20_000)
    t = np.repeat(t0[::16], 16, axis=0)                 # one target per group of 16
    keep = np.linalg.norm(r1 - t, axis=1) >= 4.5 * np.linalg.norm(r2 - r1, axis=1)
    C, s, tc = pair32(r1, r2, t, rng)
    ok = keep & (tc > F32(1e-8 * (1 + 2.5e-3)))
    sk = np.where(ok, s, F32(0))
    b = np.zeros((20_000, 3), dtype=F32)
    Cg, sg = C.reshape(20_000, 16, 3), sk.reshape(20_000, 16)
    for j in range(16):                                  # b = fma(C, s, b)
        for c in range(3):
            b[:, c] = fma32(Cg[:, j, c], sg[:, j], b[:, c])
    got = F4PI * b.astype(np.float64)
    v64 = np.where(ok[:, None], seg64(r1, r2, t), 0.0).reshape(20_000, 16, 3).sum(axis=1)
    unit = np.where(ok, F4PI * np.linalg.norm(r2 - r1, axis=1) / np.sum((r1 - t) ** 2, axis=1), 0.0)
    unit_sum = unit.reshape(20_000, 16).sum(axis=1)
    E = 256 * U * unit_sum
    err = np.linalg.norm(got - v64, axis=1)
    assert np.all(err <= E), (err / np.maximum(E, 1e-300)).max()
    # the errors are real: a bound of 8u would be broken (the worst group
    # reaches about 12u), so the test would catch a constant cut too far
    assert (err / (U * np.maximum(unit_sum, 1e-300))).max() > 8
