"""GPU: eliminate_small_loops (ov_eliminate_small_loops) against the
reference's own (oracle/_ref): the same nodes emptied and the same links
left, on rings of 3 to 40 nodes with shuffled slots and EMPTY holes, on
lines pinned to a wall, and with the origin, z-axis and outer removals
switched on.
"""
import ctypes as C

import numpy as np
import pytest

from openvort_b200 import geometry as G
from openvort_b200.tangle import EMPTY, Flow, Params
from oracle.oracle import Ref

pytestmark = pytest.mark.gpu

PARAMS = Params(vn=Flow("no flow"), vs=Flow("no flow"))
LOOP_GLOBALS = [("global_eliminate_origin_loops", C.c_int), ("global_eliminate_loops_origin_cutoff", C.c_double),
                ("global_eliminate_zaxis_loops", C.c_int), ("global_eliminate_loops_zaxis_cutoff", C.c_double),
                ("global_eliminate_outer_loops", C.c_int), ("global_eliminate_outer_loops_cutoff", C.c_double)]
DEFAULTS = {"global_eliminate_origin_loops": 0, "global_eliminate_loops_origin_cutoff": 3e-2,
            "global_eliminate_zaxis_loops": 0, "global_eliminate_loops_zaxis_cutoff": 2e-2,
            "global_eliminate_outer_loops": 0, "global_eliminate_outer_loops_cutoff": 1.0}


@pytest.fixture(scope="module")
def ov():
    import openvort_b200 as ov
    lib = ov.load()
    assert lib.ov_init(0) == 0, lib.ov_last_error_message()
    return ov


def set_loop_globals(libs, values):
    for lib in libs:
        for name, ct in LOOP_GLOBALS:
            ct.in_dll(lib, name).value = values[name]


def rings(seed, sizes, centre_spread, box, boundary="open"):
    rng = np.random.default_rng(seed)
    loops = []
    for n in sizes:
        c = rng.uniform(-centre_spread, centre_spread, size=3) + (0.0 if boundary == "open" else box / 2)
        d = rng.normal(size=3)
        loops.append(G.ring_points(c, d / np.linalg.norm(d), rng.uniform(2e-3, 6e-3), n))
    lo, hi = ((-box,) * 3, (box,) * 3) if boundary == "open" else ((0,) * 3, (box,) * 3)
    return G.rings_to_tangle(loops, lo, hi, boundary, empty_slots=5)


def compare(ov, t, loop_length):
    ref = Ref()
    want = ref.eliminate_small_loops(t, PARAMS, loop_length)
    lib = ov.load()
    ov.configure(PARAMS, ov.OV_PREC_FP64)
    got = t.copy()
    nv = lib.ov_eliminate_small_loops(got.ptr(), loop_length)
    assert nv >= 0, lib.ov_last_error_message()
    assert np.array_equal(got.stat[:, 0], want.stat[:, 0])
    assert np.array_equal(got.links, want.links)
    removed = (t.stat[:, 0] != EMPTY) & (want.stat[:, 0] == EMPTY)
    return nv, int(removed.sum())


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_small_rings_match_reference(ov, seed):
    sizes = [3, 4, 5, 6, 7, 12, 40, 5, 3, 9]
    t = G.relabel_slots(rings(seed, sizes, 0.02, 0.05), seed + 10)
    set_loop_globals([ov.load(), Ref().lib], DEFAULTS)
    nv, removed = compare(ov, t, 5)
    assert nv == 5 and removed == 3 + 4 + 5 + 5 + 3


def test_pinned_lines_match_reference(ov):
    lines = [G.wall_half_ring(n=n, radius=3e-3 * (1 + i)) for i, n in enumerate([3, 4, 5, 6, 11])]
    for i, ln in enumerate(lines):
        ln.pos[:, 0] += 0.008 * i
    t = G.relabel_slots(G.join_tangles(lines, (-0.05, -0.05, 0.0), (0.05, 0.05, 0.1), "wall-1-open"), 3)
    set_loop_globals([ov.load(), Ref().lib], DEFAULTS)
    nv, removed = compare(ov, t, 5)
    assert nv == 3 and removed == 3 + 4 + 5


@pytest.mark.parametrize("which", ["origin", "zaxis", "outer"])
def test_radial_removals_match_reference(ov, which):
    t = G.relabel_slots(rings(7, [20] * 12, 0.03, 0.06), 5)
    vals = dict(DEFAULTS)
    vals[f"global_eliminate_{which}_loops"] = 1
    vals.update({"global_eliminate_loops_origin_cutoff": 0.03, "global_eliminate_loops_zaxis_cutoff": 0.02,
                 "global_eliminate_outer_loops_cutoff": 0.025})
    set_loop_globals([ov.load(), Ref().lib], vals)
    try:
        nv, removed = compare(ov, t, 5)
        assert 0 < nv < 12
    finally:
        set_loop_globals([ov.load(), Ref().lib], DEFAULTS)
