"""GPU: vortex-vortex reconnection with the GPU pair search
(ov_reconnect_candidates, ov_reconnect_vortices) against the reference's own
reconnect() compiled from its sources (oracle/_ref): the same links,
sit-out flags, count and velocities, on crossing rings (open box) and on
dense random tangles (open and periodic); the candidate list against a
brute-force scan of the reference's tests in numpy."""
import ctypes as C

import numpy as np
import pytest

from openvort_b200 import geometry as G
from openvort_b200.tangle import Flow, Params
from oracle.oracle import Ref, have_ref, rel_err

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not have_ref(), reason="oracle/_ref not built")]

PARAMS = Params(kappa=9.97e-4, core_a=1e-8, use_mf=1, alpha=0.1, alpha_p=0.01, hyperfriction=0,
                dl_max=1e-3, vn=Flow("simple", {"external_v": (0.1, 0.0, 0.0)}), vs=Flow("no flow"))
REC_ANGLE = 0.087


@pytest.fixture(scope="module")
def ov():
    import openvort_b200 as ov
    lib = ov.load()
    assert lib.ov_init(0) == 0, lib.ov_last_error_message()
    return ov


def crossing_rings(seed, n=200, R=1e-2):
    """ring A in the xy plane; ring B in a random plane through a point a
    fraction of a spacing off A's node at (R, 0, 0)"""
    rng = np.random.default_rng(seed)
    a = G.ring_points((0, 0, 0), (0, 0, 1), R, n)
    nb = rng.normal(size=3)
    nb /= np.linalg.norm(nb)
    u = np.cross(nb, rng.normal(size=3))
    u /= np.linalg.norm(u)
    gap = rng.uniform(0.3, 1.5) * 2 * np.pi * R / n
    P = np.array([R + gap, 0.0, 0.0])
    b = G.ring_points(P - R * u, nb, R, n)
    return G.rings_to_tangle([a, b], (-0.05,) * 3, (0.05,) * 3, "open")


def prepared(t, ref):
    """tangents, normals and velocities as the reference has them before a pass"""
    return ref.update_tangle(t, PARAMS, 0.0)


def brute_candidates(t, rec_dist, rec_angle):
    n = t.n
    st = t.stat[:, 0]
    ok = (st != -1) & (st != 1) & (st != 2)
    lo = np.array(t.struct.box.bottom_left_back.p[:])
    hi = np.array(t.struct.box.top_right_front.p[:])
    L = hi - lo
    per = np.array([t.struct.box.wall[2 * a] == 1 for a in range(3)])
    tl = np.sqrt((t.tangents ** 2).sum(axis=1))
    out = []
    for k in range(n):
        if not ok[k] or tl[k] < 0.5:
            continue
        for l in range(k + 1, n):
            if not ok[l] or t.links[k, 0] == l or t.links[k, 1] == l or tl[l] < 0.5:
                continue
            d = t.pos[l] - t.pos[k]
            w = t.pos[l].copy()
            for a in range(3):
                if per[a]:
                    if d[a] > L[a] / 2:
                        w[a] -= L[a]
                    elif d[a] < -L[a] / 2:
                        w[a] += L[a]
            if np.sqrt(((t.pos[k] - w) ** 2).sum()) > rec_dist:
                continue
            c = (t.tangents[k] @ t.tangents[l]) / tl[k] / tl[l]
            if c > np.cos(rec_angle):
                continue
            out.append((k, l))
    return out


def run_ours(ov, t, rec_dist):
    lib = ov.load()
    ov.configure(PARAMS, ov.OV_PREC_FP64)
    out = t.copy()
    out.set_images_from_library(lib)
    out.recalc[:] = 0            # reconnect() zeroes them before its wall part
    n = lib.ov_reconnect_vortices(out.ptr(), 0.0, rec_dist, REC_ANGLE)
    assert n >= 0, lib.ov_last_error_message()
    return out, n


@pytest.mark.parametrize("seed", range(6))
def test_crossing_rings_match_reference(ov, seed):
    ref = Ref()
    t = prepared(crossing_rings(seed), ref)
    rec_dist = 2 * 2 * np.pi * 1e-2 / 200
    want, nw = ref.reconnect(t, PARAMS, 0.0, rec_dist, REC_ANGLE)
    got, ng = run_ours(ov, t, rec_dist)
    assert ng == nw
    assert np.array_equal(got.links, want.links)
    assert np.array_equal(got.recalc, want.recalc)
    # the velocities update_velocity wrote at each test, per node |dv| / |v|
    # (a component-wise bound is ill-posed where a component is near zero)
    assert rel_err(got.vels, want.vels, t.active) < 1e-12


@pytest.mark.parametrize("boundary", ["open", "periodic-26"])
def test_dense_tangle_matches_reference(ov, boundary):
    ref = Ref()
    D = 0.05
    t = G.random_ring_tangle(17, 40, D, dl=D / 100, boundary=boundary)
    t = prepared(t, ref)
    rec_dist = 2.5 * D / 100
    lib = ov.load()
    pairs = np.zeros(2 * 100000, np.int32)
    ov.configure(PARAMS, ov.OV_PREC_FP64)
    t.set_images_from_library(lib)
    m = lib.ov_reconnect_candidates(t.ptr(), rec_dist, REC_ANGLE, pairs.ctypes.data, 100000)
    assert m >= 0, lib.ov_last_error_message()
    cand = [tuple(p) for p in pairs[:2 * m].reshape(-1, 2)]
    assert cand == brute_candidates(t, rec_dist, REC_ANGLE)
    want, nw = ref.reconnect(t, PARAMS, 0.0, rec_dist, REC_ANGLE)
    got, ng = run_ours(ov, t, rec_dist)
    assert nw > 0, "the workload should reconnect somewhere"
    assert ng == nw
    assert np.array_equal(got.links, want.links)
    assert np.array_equal(got.recalc, want.recalc)
    # the velocities update_velocity wrote at each test, per node |dv| / |v|
    # (a component-wise bound is ill-posed where a component is near zero)
    assert rel_err(got.vels, want.vels, t.active) < 1e-12


def test_sit_out_flags_are_read_on_entry(ov):
    """Nodes flagged before the loop (by the wall part of reconnect) sit the
    pass out.  Pinned nodes sit it out the same way and change no other
    node's velocity (src/tangle.c:586-590), so the reference's pass with the
    flagged nodes pinned gives the same links and count."""
    from openvort_b200.tangle import PINNED
    ref = Ref()
    t = prepared(crossing_rings(5), ref)   # two reconnections
    rec_dist = 2 * 2 * np.pi * 1e-2 / 200
    lib = ov.load()
    base, n0 = run_ours(ov, t, rec_dist)
    assert n0 > 0
    out = t.copy()
    out.set_images_from_library(lib)
    out.recalc[:] = 1
    assert lib.ov_reconnect_vortices(out.ptr(), 0.0, rec_dist, REC_ANGLE) == 0
    assert np.array_equal(out.links, t.links)
    flagged = np.nonzero(np.any(base.links != t.links, axis=1))[0][:3]
    pinned = t.copy()
    pinned.stat[flagged, 0] = PINNED
    want, nw = ref.reconnect(pinned, PARAMS, 0.0, rec_dist, REC_ANGLE)
    out = t.copy()
    out.set_images_from_library(lib)
    out.recalc[:] = 0
    out.recalc[flagged] = 1
    ng = lib.ov_reconnect_vortices(out.ptr(), 0.0, rec_dist, REC_ANGLE)
    assert ng == nw
    assert np.array_equal(out.links, want.links)
    assert not np.array_equal(out.links, base.links)


def run_ours_mixed(ov, t, rec_dist, margin_scale=None):
    """the pass in the mixed form: FP32 far field with an error bound per
    node, FP64 sums again for tests whose sign the bound leaves open"""
    import os
    from openvort_b200._lib import ReconnectStats
    lib = ov.load()
    ov.configure(PARAMS, ov.OV_PREC_MIXED)
    out = t.copy()
    out.set_images_from_library(lib)
    out.recalc[:] = 0
    old = os.environ.get("OV_RECONNECT_MARGIN_SCALE")
    if margin_scale is not None:
        os.environ["OV_RECONNECT_MARGIN_SCALE"] = repr(margin_scale)
    try:
        n = lib.ov_reconnect_vortices(out.ptr(), 0.0, rec_dist, REC_ANGLE)
    finally:
        ov.configure(PARAMS, ov.OV_PREC_FP64)
        if old is None:
            os.environ.pop("OV_RECONNECT_MARGIN_SCALE", None)
        else:
            os.environ["OV_RECONNECT_MARGIN_SCALE"] = old
    assert n >= 0, lib.ov_last_error_message()
    st = ReconnectStats()
    assert lib.ov_reconnect_get_stats(C.byref(st)) == 0
    return out, n, st


def dense_case(boundary):
    ref = Ref()
    D = 0.05
    t = prepared(G.random_ring_tangle(17, 40, D, dl=D / 100, boundary=boundary), ref)
    return ref, t, 2.5 * D / 100


@pytest.mark.parametrize("boundary", ["open", "periodic-26"])
def test_mixed_pass_takes_the_reference_decisions(ov, boundary):
    """Mixed form: the same links, flags and count as the reference's FP64
    pass; the velocities written at each test within the mixed form's 1e-5."""
    ref, t, rec_dist = dense_case(boundary)
    want, nw = ref.reconnect(t, PARAMS, 0.0, rec_dist, REC_ANGLE)
    got, ng, st = run_ours_mixed(ov, t, rec_dist)
    assert nw > 0
    assert ng == nw == st.reconnections
    assert np.array_equal(got.links, want.links)
    assert np.array_equal(got.recalc, want.recalc)
    assert st.tested > 0 and st.nodes_summed > 0
    assert 0 <= st.fp64_rechecks <= st.tested
    assert rel_err(got.vels, want.vels, t.active) < 1e-5


@pytest.mark.parametrize("seed", range(6))
def test_mixed_pass_crossing_rings(ov, seed):
    ref = Ref()
    t = prepared(crossing_rings(seed), ref)
    rec_dist = 2 * 2 * np.pi * 1e-2 / 200
    want, nw = ref.reconnect(t, PARAMS, 0.0, rec_dist, REC_ANGLE)
    got, ng, st = run_ours_mixed(ov, t, rec_dist)
    assert ng == nw
    assert np.array_equal(got.links, want.links)
    assert np.array_equal(got.recalc, want.recalc)
    assert rel_err(got.vels, want.vels, t.active) < 1e-5


def test_mixed_pass_fp64_rechecks(ov):
    """A margin scaled beyond every |dx . dv| sends each test whose nodes
    still carry mixed sums to the FP64 re-check: the decisions stay the
    reference's and every velocity written is the FP64 one."""
    ref, t, rec_dist = dense_case("periodic-26")
    want, nw = ref.reconnect(t, PARAMS, 0.0, rec_dist, REC_ANGLE)
    got, ng, st = run_ours_mixed(ov, t, rec_dist, margin_scale=1e300)
    assert ng == nw
    assert np.array_equal(got.links, want.links)
    assert st.fp64_rechecks > 0
    assert rel_err(got.vels, want.vels, t.active) < 1e-12
