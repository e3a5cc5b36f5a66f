"""GPU: remesh and enforce_boundaries (ov_remesh, ov_enforce_boundaries)
against the reference's own remesh and enforce_boundaries (oracle/_ref),
node for node: the same nodes removed and added in the same slots, the same
links and next_free, positions, dxi, tangents and normals to rounding.

Workloads: rings whose nodes were pushed along the line (short segments:
removals) or taken out in pairs (long segments: additions), open and
periodic; a ring resolved far too finely and one far too coarsely (chains of
dependent changes); a half ring pinned to a wall.
"""
import numpy as np
import pytest

from openvort_b200 import geometry as G
from openvort_b200.tangle import EMPTY, Flow, HostTangle, Params
from oracle.oracle import Ref

pytestmark = pytest.mark.gpu

D = 0.05
DL = D / 100
MIN, MAX = 0.6 * DL, 2.5 * DL
# add_point places a node on the circle through its neighbours when the mean
# curvature is below max_curvature_scale / dl_max (1000 /cm here), else at
# their midpoint: the rings below take both branches
PARAMS = Params(dl_max=2e-4, vn=Flow("no flow"), vs=Flow("no flow"))


@pytest.fixture(scope="module")
def ov():
    import openvort_b200 as ov
    lib = ov.load()
    assert lib.ov_init(0) == 0, lib.ov_last_error_message()
    return ov


def with_empty(t, extra):
    """t with `extra` EMPTY slots appended."""
    n = len(t.pos)
    pos = np.concatenate([t.pos, np.zeros((extra, 3))])
    fwd = np.concatenate([t.links[:, 0], -np.ones(extra, np.int32)])
    rev = np.concatenate([t.links[:, 1], -np.ones(extra, np.int32)])
    st = np.concatenate([t.stat[:, 0], np.full(extra, EMPTY, np.int32)])
    pin = np.concatenate([t.stat[:, 1], -np.ones(extra, np.int32)])
    out = HostTangle(pos, fwd, rev, st, pin, t.box_lo, t.box_hi, t.boundary)
    assert len(out.pos) == n + extra
    return out


def perturb(t, seed, frac_move=0.05, n_gaps=6):
    return G.perturb_spacing(t, seed, frac_move, n_gaps)


def prepared(t, ref):
    return ref.update_tangents_normals(t, PARAMS)


def run_ours(ov, t):
    lib = ov.load()
    ov.configure(PARAMS, ov.OV_PREC_FP64)
    out = t.copy()
    out.struct.next_free = t.struct.next_free
    n = lib.ov_remesh(out.ptr(), MIN, MAX, None)
    assert n >= 0, lib.ov_last_error_message()
    return out, n


def check_same(got, want):
    assert len(got.pos) == len(want.pos)
    assert np.array_equal(got.stat[:, 0], want.stat[:, 0])
    live = want.stat[:, 0] != EMPTY
    assert np.array_equal(got.stat[live, 1], want.stat[live, 1])
    assert np.array_equal(got.links, want.links)
    assert got.struct.next_free == want.struct.next_free
    # a merged node moves by (t0 - t1) l / 2 + (n0 + n1) l^2 / 16, from
    # tangents and normals that agree with the reference's to ~1e-12
    scale = np.max(np.abs(want.pos[live]))
    assert np.max(np.abs(got.pos[live] - want.pos[live])) <= 1e-13 * scale
    assert np.max(np.abs(got.dxi[live] - want.dxi[live])) <= 1e-11 * DL

    def rel(a, b):
        return np.max(np.linalg.norm(a[live] - b[live], axis=1)) / np.max(np.linalg.norm(b[live], axis=1))

    assert rel(got.tangents, want.tangents) < 1e-10
    assert rel(got.normals, want.normals) < 1e-9


@pytest.mark.parametrize("boundary,seed", [("open", 1), ("open", 2), ("periodic-26", 3), ("periodic-26", 4)])
def test_remesh_matches_reference(ov, boundary, seed):
    ref = Ref()
    t = G.random_ring_tangle(seed, 30, D, dl=DL, boundary=boundary, empty_slots=40)
    t = prepared(perturb(t, seed), ref)
    want = ref.remesh(t, PARAMS, MIN, MAX)
    got, n = run_ours(ov, t)
    assert n > 0
    assert np.sum(want.stat[:, 0] != t.stat[:, 0]) > 0, "the workload should change something"
    check_same(got, want)


def test_remesh_chains_of_changes(ov):
    """A ring at 0.3 DL spacing (every node a removal candidate, each removal
    moving the next node) and one at 3 DL (an addition after every node, new
    slots both before and after the node being visited)."""
    ref = Ref()
    fine = G.ring_points((0.02, 0.02, 0.02), (0, 0, 1), 24 * 0.3 * DL / (2 * np.pi), 24)
    coarse = G.ring_points((0.03, 0.025, 0.02), (0.3, 0.1, 0.9), 16 * 3 * DL / (2 * np.pi), 16)
    t = G.rings_to_tangle([fine, coarse], (0, 0, 0), (D, D, D), "periodic-26", empty_slots=8)
    # empty slots before the coarse ring too
    t = with_empty(t, 16)
    t.struct.next_free = 30
    t = prepared(t, ref)
    t.struct.next_free = 30
    want = ref.remesh(t, PARAMS, MIN, MAX)
    got, n = run_ours(ov, t)
    assert n > 20
    check_same(got, want)


def test_remesh_pinned_half_ring(ov):
    ref = Ref()
    t = with_empty(G.wall_half_ring(n=48, radius=1e-2), 16)
    t = prepared(perturb(t, 8, frac_move=0.15, n_gaps=2), ref)
    p = PARAMS
    lo = 0.6 * np.pi * 1e-2 / 47
    hi = 2.5 * np.pi * 1e-2 / 47
    want = ref.remesh(t, p, lo, hi)
    lib = ov.load()
    ov.configure(p, ov.OV_PREC_FP64)
    got = t.copy()
    assert lib.ov_remesh(got.ptr(), lo, hi, None) > 0, lib.ov_last_error_message()
    check_same(got, want)


def test_remesh_without_a_free_slot_fails(ov, monkeypatch):
    monkeypatch.setenv("OV_QUIET", "1")
    ref = Ref()
    coarse = G.ring_points((0.02, 0.02, 0.02), (0, 0, 1), 16 * 3 * DL / (2 * np.pi), 16)
    t = prepared(G.rings_to_tangle([coarse], (0, 0, 0), (D, D, D), "open"), ref)
    lib = ov.load()
    ov.configure(PARAMS, ov.OV_PREC_FP64)
    assert lib.ov_remesh(t.copy().ptr(), MIN, MAX, None) == -ov._lib.OV_ERR_INVALID
    lib.ov_clear_error()


def test_remesh_nothing_to_do_changes_nothing(ov):
    ref = Ref()
    t = prepared(G.random_ring_tangle(5, 10, D, dl=DL, boundary="periodic-26"), ref)
    got, n = run_ours(ov, t)
    assert n == 0
    assert np.array_equal(got.pos, t.pos) and np.array_equal(got.links, t.links)


@pytest.mark.parametrize("boundary", ["periodic-26", "periodic-z-open-xy"])
def test_enforce_boundaries_matches_reference(ov, boundary):
    """Nodes up to three box lengths outside, through periodic and (for
    periodic-z) open faces: the reference moves a node only when the last
    failing face test names a periodic face."""
    ref = Ref()
    t = G.random_ring_tangle(9, 20, D, dl=DL, boundary=boundary)
    rng = np.random.default_rng(9)
    act = np.nonzero(t.active)[0]
    for k in rng.choice(act, size=len(act) // 4, replace=False):
        t.pos[k] += rng.integers(-3, 4, size=3) * D + rng.uniform(-0.01, 0.01, size=3) * D
    want = ref.enforce_boundaries(t, PARAMS)
    lib = ov.load()
    ov.configure(PARAMS, ov.OV_PREC_FP64)
    got = t.copy()
    moved = lib.ov_enforce_boundaries(got.ptr())
    assert moved > 0, lib.ov_last_error_message()
    assert np.array_equal(got.pos[t.active], want.pos[t.active])
    assert moved == int(np.sum(np.any(want.pos[t.active] != t.pos[t.active], axis=1)))


def test_empty_tangles(ov):
    """N = 0 and a tangle of EMPTY slots only: nothing to do, no error."""
    from openvort_b200.tangle import HostTangle
    lib = ov.load()
    ov.configure(PARAMS, ov.OV_PREC_FP64)
    for n in (0, 5):
        st = np.full(n, EMPTY, np.int32)
        t = HostTangle(np.zeros((n, 3)), -np.ones(n, np.int32), -np.ones(n, np.int32), st, -np.ones(n, np.int32),
                       (0, 0, 0), (D, D, D), "periodic-26")
        assert lib.ov_remesh(t.ptr(), MIN, MAX, None) == 0, lib.ov_last_error_message()
        assert lib.ov_enforce_boundaries(t.ptr()) == 0
        assert lib.ov_eliminate_small_loops(t.ptr(), 5) == 0
        assert lib.ov_reconnect_vortices(t.ptr(), 0.0, 1e-3, 0.087) == 0, lib.ov_last_error_message()
        assert lib.ov_reconnect_candidates(t.ptr(), 1e-3, 0.087, None, 0) == 0
        assert np.all(t.stat[:, 0] == EMPTY)
