"""GPU: frames from a device-resident state (ov_state_save_frame).

The frame is the state at the call: steps taken while the file is being
written do not reach it.  Text frames equal ov_save_tangle of the state
downloaded at that moment (which equals the reference's save_tangle, see
test_frames.py); binary frames load back to the same arrays and time.
"""
import ctypes as C

import numpy as np
import pytest

from openvort_b200 import _lib, geometry as G
from openvort_b200.tangle import Flow, HostTangle, Params

pytestmark = pytest.mark.gpu

PARAMS = Params(use_mf=1, alpha=0.098, alpha_p=0.016, vn=Flow("simple", {"external_v": (0.5, 0, 0)}),
                vs=Flow("no flow"), dl_max=1e-3)


@pytest.fixture(scope="module")
def ov():
    import openvort_b200 as ov
    lib = ov.load()
    assert lib.ov_init(0) == 0, lib.ov_last_error_message()
    return ov


def blank_like(t):
    n = len(t.pos)
    return HostTangle(np.zeros((n, 3)), np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n, np.int32),
                      np.zeros(n, np.int32), (0, 0, 0), (1, 1, 1), "open")


@pytest.mark.parametrize("binary", [False, True])
def test_state_frame_is_the_state_at_the_call(ov, tmp_path, binary):
    ov.configure(PARAMS, ov.OV_PREC_FP64)
    t = G.random_ring_tangle(12, 40, 0.05, dl=5e-4, boundary="periodic-26", empty_slots=9)
    st = ov.DeviceState(t)
    st.update_tangle(0.0)
    st.download()
    snap = t.copy()
    for name in ("vels", "tangents", "normals", "dxi"):
        getattr(snap, name)[:] = getattr(t, name)
    path = tmp_path / ("f.bin" if binary else "f.dat")
    st.save_frame(path, 0.5, binary=binary)
    for k in range(3):           # the state moves on while the file is written
        st.rk4_step(k * 1e-5, 1e-5)
    st.wait_frames()
    st.download()
    assert not np.array_equal(t.pos, snap.pos)
    lib = ov.load()
    if binary:
        back = blank_like(t)
        tm = C.c_double(0)
        assert lib.ov_load_frame(str(path).encode(), back.ptr(), C.byref(tm)) == 0, lib.ov_last_error_message()
        assert tm.value == 0.5
        live = t.active
        for name in ("pos", "vels", "tangents", "normals", "dxi"):
            assert np.array_equal(getattr(back, name)[live], getattr(snap, name)[live]), name
        assert np.array_equal(back.links, snap.links) and np.array_equal(back.stat, snap.stat)
        assert list(back.struct.box.wall) == list(t.struct.box.wall)
    else:
        want = tmp_path / "want.dat"
        assert lib.ov_save_tangle(snap.ptr(), str(want).encode()) == 0
        assert path.read_bytes() == want.read_bytes()
    st.close()


def test_frames_of_several_states_and_back_to_back(ov, tmp_path):
    ov.configure(PARAMS, ov.OV_PREC_FP64)
    a = ov.DeviceState(G.random_ring_tangle(1, 10, 0.05, dl=5e-4, boundary="periodic-26"))
    b = ov.DeviceState(G.random_ring_tangle(2, 12, 0.05, dl=5e-4, boundary="periodic-26"))
    a.update_tangle(0.0)
    b.update_tangle(0.0)
    for i in range(3):
        a.save_frame(tmp_path / f"a{i}.bin", float(i))
        b.save_frame(tmp_path / f"b{i}.bin", float(i))
        a.rk4_step(0.0, 1e-5)
        b.rk4_step(0.0, 1e-5)
    a.wait_frames()
    lib = ov.load()
    for i in range(3):
        for s, t in (("a", a.t), ("b", b.t)):
            n, tm = C.c_int(0), C.c_double(0)
            assert lib.ov_frame_info(str(tmp_path / f"{s}{i}.bin").encode(), C.byref(n), C.byref(tm)) == 0
            assert n.value == len(t.pos) and tm.value == float(i)
    a.close()
    b.close()
