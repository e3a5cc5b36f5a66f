"""GPU: batched ensembles of independent open-boundary systems (ov_batch_*).

Every system must evolve exactly as a tangle of its own would: velocities and
RK4 positions of each system against the CPU oracle run on that system
alone (FP64 path: 1e-12 on velocities, 1e-14 on positions relative to the
step's displacement scale), the mixed form against the FP64 form (1e-5), the
CUDA-graph run against step-by-step single-tangle runs, and the autotuned
kernel shape against the default one.
"""
import dataclasses

import numpy as np
import pytest

from cases import pos_err, rel_err
from openvort_b200 import geometry as G
from openvort_b200.tangle import Flow, Params
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

TOL_V64, TOL_MIXED = 1e-12, 1e-5

PARAMS = Params(kappa=9.97e-4, core_a=1e-8, use_mf=1, alpha=0.098, alpha_p=0.016,
                hyperfriction=1, max_curv_scale=0.2, hyperalpha=0.5, dl_max=1e-3,
                vn=Flow("simple", {"external_v": (0.2, 0.0, 0.0)}), vs=Flow("no flow"))


@pytest.fixture(scope="module")
def ov():
    import openvort_b200 as ov
    lib = ov.load()
    assert lib.ov_init(0) == 0, lib.ov_last_error_message()
    return ov


@pytest.fixture(scope="module")
def ensemble():
    return G.ring_pair_ensemble(7, 6, n_range=(64, 400))


def system_tangle(rings):
    half = 0.09
    return G.rings_to_tangle(rings, (-half,) * 3, (half,) * 3, "open")


def test_batch_update_fp64_vs_oracle(ov, ensemble):
    t, off, systems = ensemble
    ov.configure(PARAMS, ov.OV_PREC_FP64)
    b = ov.DeviceBatch(t.copy(), off)
    b.update(0.0)
    b.download()
    orc = Oracle()
    for s, rings in enumerate(systems):
        ref = orc.update_tangle(system_tangle(rings), PARAMS, 0.0)
        sl = slice(off[s], off[s + 1])
        assert rel_err(b.t.vels[sl], ref.vels) < TOL_V64, s
        assert rel_err(b.t.vs[sl], ref.vs) < TOL_V64, s
    b.close()


def test_batch_mixed_vs_fp64(ov, ensemble):
    t, off, _ = ensemble
    out = {}
    for prec in (ov.OV_PREC_FP64, ov.OV_PREC_MIXED):
        ov.configure(PARAMS, prec)
        b = ov.DeviceBatch(t.copy(), off)
        b.update(0.0)
        b.download()
        out[prec] = b.t.vels.copy()
        b.close()
    ov.configure(PARAMS, ov.OV_PREC_FP64)
    assert rel_err(out[ov.OV_PREC_MIXED], out[ov.OV_PREC_FP64]) < TOL_MIXED


def test_batch_graph_run_vs_oracle_rk4(ov, ensemble):
    t, off, systems = ensemble
    dt, steps = 2e-5, 3
    ov.configure(PARAMS, ov.OV_PREC_FP64)
    b = ov.DeviceBatch(t.copy(), off)
    b.run(0.0, dt, steps)
    b.download()
    st = b.stats()
    assert st.evals == 4 * steps and st.kernels_per_step > 0
    orc = Oracle()
    for s, rings in enumerate(systems):
        cur = system_tangle(rings)
        tt = 0.0
        for _ in range(steps):
            cur = orc.update_tangle(cur, PARAMS, tt)
            cur = orc.rk4_step(cur, PARAMS, tt, dt)
            tt += dt
        sl = slice(off[s], off[s + 1])
        assert pos_err(b.t.pos[sl], cur.pos) < 1e-14, s
    b.close()


def test_batch_matches_single_tangle_states(ov, ensemble):
    """The same system through ov_state_run and through the batch."""
    t, off, systems = ensemble
    ov.configure(PARAMS, ov.OV_PREC_MIXED)
    b = ov.DeviceBatch(t.copy(), off)
    b.run(0.0, 1e-5, 2)
    b.download()
    for s in (0, len(systems) - 1):
        st = ov.DeviceState(system_tangle(systems[s]))
        st.run(0.0, 1e-5, 2)
        st.download()
        sl = slice(off[s], off[s + 1])
        x0 = system_tangle(systems[s]).pos
        # both are mixed runs (with different near radii): the displacements
        # agree within the mixed tolerance
        assert rel_err(b.t.pos[sl] - x0, st.t.pos - x0) < TOL_MIXED
        assert rel_err(b.t.vels[sl], st.t.vels) < TOL_MIXED
        st.close()
    b.close()
    ov.configure(PARAMS, ov.OV_PREC_FP64)


def test_batch_graph_replays_are_deterministic(ov, ensemble):
    t, off, _ = ensemble
    ov.configure(PARAMS, ov.OV_PREC_MIXED)
    a = ov.DeviceBatch(t.copy(), off)
    a.run(0.0, 1e-5, 4)
    a.download()
    c = ov.DeviceBatch(t.copy(), off)
    c.run(0.0, 1e-5, 2)
    c.run(2e-5, 1e-5, 2)
    c.download()
    assert np.array_equal(a.t.pos, c.t.pos)
    a.close()
    c.close()
    ov.configure(PARAMS, ov.OV_PREC_FP64)


def test_batch_autotune_keeps_results(ov, ensemble):
    t, off, _ = ensemble
    ov.configure(PARAMS, ov.OV_PREC_MIXED)
    b = ov.DeviceBatch(t.copy(), off)
    b.update(0.0)
    b.download()
    v0 = b.t.vels.copy()
    tu = b.autotune()
    assert tu.targets_per_block in (64, 128, 256) and tu.sources_per_tile in (0, 64, 128, 256)
    assert tu.kernel_ms > 0
    b.update(0.0)
    b.download()
    # the FP32 offsets are taken from each block's first target, so another
    # shape rounds differently: within the mixed tolerance
    assert rel_err(b.t.vels, v0) < TOL_MIXED
    # FP64: every shape sums a target's sources in the same order
    ov.configure(PARAMS, ov.OV_PREC_FP64)
    b.update(0.0)
    b.download()
    v64 = b.t.vels.copy()
    for shape in ((64, 64), (256, 256), (128, 64), (128, 0)):
        b.set_tuning(*shape)
        b.update(0.0)
        b.download()
        assert np.array_equal(b.t.vels, v64)
    b.close()


@pytest.mark.parametrize("tb", [64, 128, 256])
def test_batch_chain_order_mixed_vs_fp64(ov, ensemble, tb):
    """The chain-order mixed kernel (sources_per_tile 0) within the mixed
    tolerance of the FP64 sums."""
    t, off, _ = ensemble
    ov.configure(PARAMS, ov.OV_PREC_FP64)
    b = ov.DeviceBatch(t.copy(), off)
    b.update(0.0)
    b.download()
    v64 = b.t.vels.copy()
    b.close()
    ov.configure(PARAMS, ov.OV_PREC_MIXED)
    b = ov.DeviceBatch(t.copy(), off)
    b.set_tuning(tb, 0)
    b.update(0.0)
    b.download()
    assert rel_err(b.t.vels, v64) < TOL_MIXED
    b.close()
    ov.configure(PARAMS, ov.OV_PREC_FP64)


def test_batch_rejects_bad_ensembles(ov, ensemble, monkeypatch):
    monkeypatch.setenv("OV_QUIET", "1")
    t, off, _ = ensemble
    lib = ov.load()
    ov.configure(PARAMS, ov.OV_PREC_FP64)
    bad = t.copy()
    bad.links[int(off[1]), 0] = int(off[2])      # a link into the next system
    bad._bind()
    assert not lib.ov_batch_create(bad.ptr(), len(off) - 1, off.ctypes.data)
    assert lib.ov_last_error() == ov._lib.OV_ERR_INVALID
    lib.ov_clear_error()
    wrong = off.copy()
    wrong[-1] += 1
    assert not lib.ov_batch_create(t.ptr(), len(off) - 1, wrong.ctypes.data)
    assert lib.ov_last_error() == ov._lib.OV_ERR_INVALID
    lib.ov_clear_error()
    per = G.rings_to_tangle([G.ring_points((0.05, 0.05, 0.05), (0, 0, 1), 0.01, 64)],
                            (0, 0, 0), (0.1, 0.1, 0.1), "periodic-6")
    two = np.array([0, per.n], np.int32)
    assert not lib.ov_batch_create(per.ptr(), 1, two.ctypes.data)
    assert lib.ov_last_error() == ov._lib.OV_ERR_INVALID
    lib.ov_clear_error()
