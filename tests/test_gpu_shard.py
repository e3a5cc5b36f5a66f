"""One tangle sharded over ranks (ov_state_shard*), on one GPU.

W device states in one process stand for W ranks.  Each walks only its
share of the targets, a contiguous range of the tree's key order.  Between
shard_begin and shard_end the test copies every rank's block into the
others' exchange buffers, which is what the all-gather of a multi-GPU run
does.  Every rank's state must then equal a single ov_state_run bit for bit,
in both precisions.  The multi-process exchange itself is tested with gloo
in test_dist.py."""
import numpy as np
import pytest

from openvort_b200 import geometry as G
from openvort_b200.tangle import Flow, Params

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

DT = 1e-6


@pytest.fixture(scope="module")
def ov():
    import openvort_b200 as ov
    lib = ov.load()
    assert lib.ov_init(0) == 0, lib.ov_last_error_message()
    return ov


def tangle_and_params(use_bh=1):
    t = G.random_ring_tangle(17, 60, 0.1, boundary="periodic-26", empty_slots=5)
    p = Params(core_a=1e-8, alpha=0.098, alpha_p=0.016, use_mf=1, dl_max=1e-3, use_bh=use_bh,
               bh_theta=0.5, vn=Flow("simple", {"external_v": (0.5, 0, 0)}))
    return t, p


def run_ranks(ov, t, world, steps, own_buffer=False):
    """`steps` sharded RK4 steps of `world` emulated ranks; their states."""
    states, bufs = [], []
    for r in range(world):
        st = ov.DeviceState(t.copy())
        if own_buffer:
            st.shard(r, world, None, 0)
        else:
            nb = st.shard_bytes(world)
            xb = torch.zeros(nb // 8, dtype=torch.float64, device="cuda")
            st.shard(r, world, xb.data_ptr(), nb)
            st.xbuf = xb                    # alive as long as the state
            bufs.append(xb)
        states.append(st)
    block = bufs[0].numel() // world if bufs else 0
    tt = 0.0
    for _ in range(steps):
        for q in range(4):
            for st in states:
                st.shard_begin(q, tt, DT)
            for r in range(len(bufs)):
                for o in range(len(bufs)):
                    if o != r:
                        bufs[o][r * block:(r + 1) * block].copy_(bufs[r][r * block:(r + 1) * block])
            torch.cuda.synchronize()
            for st in states:
                st.shard_end(q, tt, DT)
        tt += DT
    for st in states:
        st.download()
    return states


@pytest.mark.parametrize("precision", [0, 1])
def test_sharded_steps_with_nodes_outside_the_box(ov, precision):
    """Nodes just outside the root box sort last in the key order, so the
    last rank's share holds them, and its walk gives each a warp of its own:
    3 ranks still equal one run bit for bit."""
    t, p = tangle_and_params()
    a = np.nonzero(t.active)[0]
    for ax in range(3):
        k = a[np.argmin(t.pos[a, ax])]
        t.pos[k, ax] = -1e-6
        k = a[np.argmax(t.pos[a, ax])]
        t.pos[k, ax] = 0.1 + 1e-6
    ov.configure(p, precision)
    ref = ov.DeviceState(t.copy())
    ref.run(0.0, DT, 2)
    ref.download()
    act = t.active
    for st in run_ranks(ov, t, 3, 2):
        assert np.array_equal(st.t.pos[act], ref.t.pos[act])


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("world", [1, 3])
def test_sharded_steps_equal_one_run(ov, precision, world):
    t, p = tangle_and_params()
    ov.configure(p, precision)
    ref = ov.DeviceState(t.copy())
    ref.run(0.0, DT, 2)
    ref.download()
    act = t.active
    for st in run_ranks(ov, t, world, 2, own_buffer=(world == 1)):
        assert np.array_equal(st.t.pos[act], ref.t.pos[act])
        assert np.array_equal(st.t.vels[act], ref.t.vels[act])
        assert np.array_equal(st.t.vs[act], ref.t.vs[act])
        st.close()
    ref.close()


def test_sharded_counters_split_the_walk(ov):
    """Each rank evaluates only its own targets: the ranks' cell
    evaluations add up to those of the whole run."""
    t, p = tangle_and_params()
    ov.configure(p, 1)
    ref = ov.DeviceState(t.copy())
    ref.reset_stats()
    ref.run(0.0, DT, 1)
    whole = ref.stats().cell_interactions
    states = run_ranks(ov, t, 3, 1)
    parts = [st.stats().cell_interactions for st in states]
    assert sum(parts) == whole
    assert all(0 < x < whole for x in parts)
    for st in states:
        st.close()
    ref.close()


def test_shard_errors(ov, monkeypatch):
    monkeypatch.setenv("OV_QUIET", "1")
    t, p = tangle_and_params(use_bh=0)
    ov.configure(p, 0)
    st = ov.DeviceState(t.copy())
    with pytest.raises(ov.OVError):
        st.shard(3, 3, None, 0)             # rank beyond the world
    with pytest.raises(ov.OVError):
        st.shard(0, 2, None, 0)             # several ranks need a buffer
    xb = torch.zeros(8, dtype=torch.float64, device="cuda")
    with pytest.raises(ov.OVError):
        st.shard(0, 2, xb.data_ptr(), 64)   # too small for the tangle
    with pytest.raises(ov.OVError):
        st.shard_begin(0, 0.0, DT)          # no buffer set yet
    st.shard(0, 1, None, 0)
    with pytest.raises(ov.OVError):
        st.shard_begin(0, 0.0, DT)          # the direct sum is not sharded
    with pytest.raises(ov.OVError):
        st.shard_begin(4, 0.0, DT)          # stages are 0..3
    st.close()


def test_more_ranks_than_nodes(ov):
    """8 ranks over a 5-node loop: ranks 5..7 own no targets, and every
    rank still ends with the one-GPU state."""
    from openvort_b200.tangle import ring_points
    r = ring_points(np.array([0.05, 0.05, 0.05]), (0.3, 0.2, 0.9), 0.004, 5)
    t = G.rings_to_tangle([r], (0, 0, 0), (0.1, 0.1, 0.1), "periodic-26", empty_slots=3)
    p = Params(core_a=1e-8, alpha=0.098, alpha_p=0.016, use_mf=1, dl_max=1e-2, use_bh=1, bh_theta=0.5)
    ov.configure(p, 0)
    ref = ov.DeviceState(t.copy())
    ref.run(0.0, DT, 2)
    ref.download()
    for st in run_ranks(ov, t, 8, 2):
        assert np.array_equal(st.t.pos[t.active], ref.t.pos[t.active])
        st.close()
    ref.close()
