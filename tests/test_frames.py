"""Frame files on the host (no GPU needed: writing a frame is I/O).

ov_save_tangle writes the reference's save_tangle text frames byte for
byte; the comparison runs the reference's own save_tangle (oracle/_ref) on
the same tangles: rings with EMPTY holes, an open line pinned to a wall, and
tangles whose slots are shuffled so that vortices start mid-array and slot
0 sits inside a line.  Binary frames round-trip every slot array, the box,
the walls and the time.
"""
import ctypes as C

import numpy as np
import pytest

from openvort_b200 import _lib, geometry as G
from openvort_b200.tangle import HostTangle
from oracle.oracle import Ref, have_ref


@pytest.fixture(scope="module")
def lib():
    if not _lib.LIB_PATH.exists():
        from openvort_b200 import build
        build.build()
    return _lib.load()


def filled(t, seed):
    """Values of every magnitude and sign in the per-node arrays."""
    rng = np.random.default_rng(seed)
    n = len(t.pos)
    scale = 10.0 ** rng.integers(-12, 6, size=(n, 3))
    t.vels[:] = rng.normal(size=(n, 3)) * scale
    t.tangents[:] = rng.normal(size=(n, 3))
    t.normals[:] = rng.normal(size=(n, 3)) * 1e3
    t.dxi[:] = rng.uniform(0, 1e-3, size=n)
    t.vels[0, 0] = -0.0
    return t


def relabel(t, seed):
    return G.relabel_slots(t, seed)


def cases():
    rings = G.random_ring_tangle(3, 12, 0.05, dl=5e-4, boundary="periodic-26", empty_slots=7)
    G.perturb_spacing(rings, 3, frac_move=0.0, n_gaps=4)
    half = G.wall_half_ring(n=40)
    yield "rings", filled(rings, 1)
    yield "half_ring", filled(half, 2)
    yield "rings_shuffled", relabel(filled(rings, 3), 4)
    yield "half_ring_shuffled", relabel(filled(half, 5), 6)
    empty0 = filled(G.random_ring_tangle(8, 3, 0.05, dl=5e-4, boundary="open", empty_slots=2), 7)
    yield "empty_slot_0", relabel(empty0, 9)


@pytest.mark.skipif(not have_ref(), reason="reference library not built")
@pytest.mark.parametrize("name,t", list(cases()))
def test_text_frame_is_the_reference_file(lib, tmp_path, name, t):
    ref = Ref()
    ours, theirs = tmp_path / "ours.dat", tmp_path / "ref.dat"
    assert lib.ov_save_tangle(t.ptr(), str(ours).encode()) == 0, lib.ov_last_error_message()
    f = ref.lib.save_tangle
    f.restype = None
    f.argtypes = [C.c_char_p, C.c_void_p]
    f(str(theirs).encode(), C.cast(t.ptr(), C.c_void_p))
    a, b = ours.read_bytes(), theirs.read_bytes()
    assert len(a) > 0
    assert a == b


def test_binary_frame_round_trip(lib, tmp_path):
    t = filled(G.random_ring_tangle(4, 6, 0.05, dl=5e-4, boundary="periodic-26", empty_slots=5), 11)
    path = str(tmp_path / "f.bin").encode()
    assert lib.ov_save_frame(t.ptr(), path, 0.125, _lib.OV_FRAME_BINARY) == 0, lib.ov_last_error_message()
    n, time = C.c_int(0), C.c_double(0)
    assert lib.ov_frame_info(path, C.byref(n), C.byref(time)) == 0
    assert n.value == len(t.pos) and time.value == 0.125
    back = HostTangle(np.zeros_like(t.pos), np.zeros(n.value, np.int32), np.zeros(n.value, np.int32),
                      np.zeros(n.value, np.int32), np.zeros(n.value, np.int32), (0, 0, 0), (1, 1, 1), "open")
    got_time = C.c_double(0)
    assert lib.ov_load_frame(path, back.ptr(), C.byref(got_time)) == 0, lib.ov_last_error_message()
    assert got_time.value == 0.125
    for name in ("pos", "vels", "tangents", "normals", "dxi", "links", "stat"):
        assert np.array_equal(getattr(back, name), getattr(t, name)), name
    box = back.struct.box
    assert [box.bottom_left_back.p[c] for c in range(3)] == list(t.box_lo)
    assert [box.top_right_front.p[c] for c in range(3)] == list(t.box_hi)
    assert list(box.wall) == list(t.struct.box.wall)


def test_load_frame_rejects_mismatches(lib, tmp_path, monkeypatch):
    monkeypatch.setenv("OV_QUIET", "1")
    t = G.random_ring_tangle(4, 2, 0.05, dl=5e-4, boundary="open")
    path = tmp_path / "f.bin"
    assert lib.ov_save_frame(t.ptr(), str(path).encode(), 0.0, _lib.OV_FRAME_BINARY) == 0
    small = G.random_ring_tangle(4, 1, 0.05, dl=5e-4, boundary="open")
    assert lib.ov_load_frame(str(path).encode(), small.ptr(), None) == -_lib.OV_ERR_INVALID
    text = tmp_path / "f.dat"
    assert lib.ov_save_tangle(filled(t, 1).ptr(), str(text).encode()) == 0
    assert lib.ov_frame_info(str(text).encode(), None, None) == -_lib.OV_ERR_INVALID
    (tmp_path / "cut.bin").write_bytes(path.read_bytes()[:-9])
    assert lib.ov_load_frame(str(tmp_path / "cut.bin").encode(), t.ptr(), None) == -_lib.OV_ERR_INVALID
    lib.ov_clear_error()
