"""The CPU oracle (oracle/ov_oracle.c) pinned against the reference: the
golden fixtures the reference produced (tests/golden/), and the reference
itself where oracle/_ref was built.  CPU only."""
import numpy as np
import pytest

from cases import NAMES, load, pos_err, rel_err
from openvort_b200 import geometry as G
from openvort_b200.tangle import FLOW_PARAMS, Flow, Params
from oracle.oracle import Oracle, Ref, have_ref

# FP64 parity bound on velocities (max over nodes of |dv| / |v_ref|)
TOL_V = 1e-12
# normals: second differences over nodes ~dl apart cancel ~3 digits, and
# the restatement factors the stencil weights differently
TOL_N = 1e-11


@pytest.fixture(scope="module")
def oracle():
    return Oracle()


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_golden(oracle, name):
    t, p, meta, z = load(name)
    out = oracle.update_tangle(t, p, meta["time"])
    act = t.active
    assert np.max(np.abs(out.dxi - z["dxi"])[act]) <= 1e-15 * np.max(z["dxi"][act])
    assert rel_err(out.tangents, z["tangents"], act) < TOL_N
    assert rel_err(out.normals, z["normals"], act) < TOL_N * 10
    assert rel_err(out.vs, z["vs"], act) < TOL_V
    assert rel_err(out.vels, z["vels"], act) < TOL_V


@pytest.mark.parametrize("name", [n for n in NAMES if "ring256" in n or "direct" in n or "bh4" in n
                                  or "flows" in n])
def test_oracle_rk4_matches_golden(oracle, name):
    t, p, meta, z = load(name)
    steps = meta["rk4_steps"]
    if steps == 0:
        pytest.skip("no RK4 steps in this fixture")
    cur = oracle.update_tangle(t, p, meta["time"])
    tt = meta["time"]
    for s in range(steps):
        nxt = oracle.rk4_step(cur, p, tt, meta["dt"])
        tt += meta["dt"]
        cur = oracle.update_tangle(nxt, p, tt)
        assert pos_err(cur.pos, z[f"rk4_pos_{s + 1}"], t.active) < 1e-14


def test_oracle_bh4_on_the_config2_tangle(oracle):
    """Barnes-Hut theta 0.4 on the 22.4k-point periodic tangle: the restated
    tree against the reference's update_velocity at 256 sample nodes."""
    from cases import cfg2_params, load_cfg2_samples
    t, z = load_cfg2_samples()
    out = oracle.update_tangle(t, cfg2_params(1))
    assert rel_err(out.vs[z["idx"]], z["vs_bh4"]) < TOL_V
    # the tree's approximation is far above the parity bound: the tree ran
    assert rel_err(z["vs_bh4"], z["vs_direct"]) > 1e-4


def test_oracle_bh4_on_another_config2_seed(oracle):
    """The same on config 2's seed 3 (64 sample nodes)."""
    from cases import cfg2_params, load_cfg2_samples
    t, z = load_cfg2_samples(3)
    out = oracle.update_tangle(t, cfg2_params(1))
    assert rel_err(out.vs[z["idx"]], z["vs_bh4"]) < TOL_V


def test_bh_differs_from_direct(oracle):
    """The Barnes-Hut fixtures exercise the tree: their error against the
    direct sum is the reference's BH error, orders above the parity bound."""
    t, pd, _, zd = load("periodic26_direct")
    for th, lo, hi in ((3, 1e-4, 1e-1), (5, 1e-3, 2e-1)):
        _, pb, _, zb = load(f"periodic26_bh{th}")
        e = rel_err(zb["vs"], zd["vs"], t.active)
        assert lo < e < hi


def test_ring_speed_thin_core(oracle):
    """Self-induced speed of a ring vs kappa/(4 pi R)(ln(8R/a) - 1/2): the
    reference's discretisation sits about +2.2 % above (python/one_loop_r.py:69)."""
    R, a, kappa = 1e-2, 1.3e-8, 9.97e-4
    t = G.single_ring(256, R)
    p = Params(core_a=a, use_mf=0, alpha=0, alpha_p=0, hyperfriction=0, dl_max=1e-3)
    out = oracle.update_tangle(t, p)
    vz = out.vels[:, 2].mean()
    v_thin = kappa / (4 * np.pi * R) * (np.log(8 * R / a) - 0.5)
    assert abs(vz / v_thin - 1) < 0.03
    assert np.std(out.vels[:, 2]) / abs(vz) < 1e-10


def test_rk4_stage4_half_step(oracle):
    """rk4_classic changes the step: the reference's stage 4 uses dt/2."""
    t, p, meta, z = load("ring256")
    cur = oracle.update_tangle(t, p)
    a = oracle.rk4_step(cur, p, 0.0, 5e-6)
    b = oracle.rk4_step(cur, p, 0.0, 5e-6, rk4_classic=True)
    assert pos_err(a.pos, z["rk4_pos_1"]) < 1e-14
    assert np.max(np.abs(a.pos - b.pos)) > 0


@pytest.mark.skipif(not have_ref(), reason="reference library not built here")
@pytest.mark.parametrize("theta,quad", [(0.2, 0), (0.45, 0), (0.4, 1)])
def test_oracle_vs_reference_live(oracle, theta, quad):
    """Fresh seeds against the compiled reference, including the quadtree."""
    ref = Ref(threads=4)
    t = G.random_ring_tangle(11, 12, 0.1, boundary="periodic-6")
    p = Params(core_a=1.3e-8, alpha=0.098, alpha_p=0.016, dl_max=1e-3, use_bh=1,
               bh_theta=theta, bh_quadtree=quad, vn=Flow("simple", {"external_v": (0.2, 0.1, 0)}))
    a = oracle.update_tangle(t, p, 0.0)
    b = ref.update_tangle(t, p, 0.0)
    assert rel_err(a.vels, b.vels, t.active) < TOL_V


@pytest.mark.skipif(not have_ref(), reason="reference library not built here")
def test_oracle_point_queries_vs_reference(oracle):
    ref = Ref(threads=4)
    t, p, _, _ = load("periodic26_bh4")
    rng = np.random.default_rng(5)
    pts = rng.uniform(0, 0.1, size=(64, 3))
    skip = rng.integers(-1, t.n, size=64).astype(np.int32)
    assert rel_err(oracle.segments_at(t, p, pts, skip), ref.segments_at(t, p, pts, skip)) < TOL_V
    assert rel_err(oracle.bh_at(t, p, pts, skip), ref.bh_at(t, p, pts, skip)) < TOL_V


def test_oracle_flows_match_reference_fixture(oracle):
    """The restated flows against the reference's update_tangle with each
    flow of its table as vn_conf and as vs_conf (flows16 fixture)."""
    import dataclasses
    from cases import fixture_flows
    t, base, meta, z = load("flows16")
    act = t.active
    for i, f in fixture_flows(meta):
        for which in ("vn", "vs"):
            out = oracle.update_tangle(t, dataclasses.replace(base, **{which: f}), meta["time"])
            assert rel_err(out.vels, z[f"vels_{which}_{i}"], act) < TOL_V, (f.name, which)


@pytest.mark.skipif(not have_ref(), reason="reference library not built here")
def test_reference_spherical_and_simple_leaves_its_output_unwritten():
    """Pins the reference's behaviour behind the library's one deviation:
    get_v_spherical_and_simple (src/external_velocity.c:226-237) returns the
    1 of get_v_simple as an error before adding the two flows, so the
    caller's vector keeps whatever it held.  Its two parts each write."""
    import ctypes as C
    from openvort_b200.tangle import Vec3d
    ref = Ref(threads=1)
    prm = {"external_v": (0.3, -0.1, 0.2), "strength": 2e-3, "cutoff": 0.02}
    where = Vec3d((0.03, 0.02, 0.01))
    for fname, fn, want_rc, writes in (("spherical and simple", "get_v_spherical_and_simple", 1, False),
                                       ("spherical", "get_v_spherical", 0, True),
                                       ("simple", "get_v_simple", 1, True)):
        conf, keep = Flow(fname, {k: v for k, v in prm.items()
                                  if k in dict(FLOW_PARAMS[fname])}).vconf()
        res = Vec3d((-7.0, -7.0, -7.0))
        f = getattr(ref.lib, fn)
        f.restype = C.c_int
        f.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]
        rc = f(C.addressof(where), 0.0, C.addressof(res), C.addressof(conf))
        assert rc == want_rc, fname
        assert (list(res.p) != [-7.0] * 3) == writes, fname


def test_flows_restated(oracle):
    """Every external flow of the reference's table evaluates (no NaN) and
    'simple' returns its vector."""
    t = G.single_ring(16, 1e-2, center=(0.03, 0.02, 0.01))
    flows = {
        "no flow": {}, "spherical": {"strength": 1e-3, "cutoff": 1e-3},
        "simple": {"external_v": (0.1, 0.2, 0.3)},
        "spherical and simple": {"external_v": (0.1, 0, 0), "strength": 1e-3, "cutoff": 1e-3},
        "cylindrical": {"strength": 1e-3, "cutoff": 1e-3},
        "oscillating": {"strength": 0.1, "frequency": 10, "wave": (1, 0, 0), "polarization": (0, 1, 0)},
        "oscillating slit": {"strength": 0.1, "frequency": 10, "cutoff": 0.01},
        "coscos": {"k": 10, "v0": 0.1, "l": 0.1}, "coscos-divfree": {"k": 10, "v0": 0.1, "l": 0.1},
        "cos-divfree": {"k": 10, "v0": 0.1, "l": 0.1}, "simple-shear": {"rate": 1.0, "v0": 0.1},
        "rotosc": {"freq": 5.0, "amp": 0.2}, "DG": {"rot": 1.0, "vz": 0.1},
        "rotosc-boundary": {"freq": 5.0, "amp": 0.2}, "constant acceleration": {"accel": 2.0},
        "parabolic": {"H": 0.1, "amp": 1.0},
    }
    for name, prm in flows.items():
        p = Params(lia_only=1, use_mf=0, hyperfriction=0, vs=Flow(name, prm))
        out = oracle.update_tangle(t, p, 0.01)
        assert np.all(np.isfinite(out.vels)), name


@pytest.mark.skipif(not have_ref(), reason="reference library not built here")
@pytest.mark.parametrize("use_bh,boundary", [(0, "periodic-26"), (1, "periodic-26"), (1, "periodic-18"),
                                             (0, "open")])
def test_oracle_vs_reference_smallest_loop(oracle, use_bh, boundary):
    """A 5-node loop among EMPTY slots (the GPU suite's smallest case): every
    stencil reaches round the loop and the tree has a handful of cells."""
    from openvort_b200.tangle import ring_points
    ref = Ref(threads=2)
    r = ring_points(np.array([0.05, 0.05, 0.05]), (0.3, 0.2, 0.9), 0.004, 5)
    t = G.rings_to_tangle([r], (0, 0, 0), (0.1, 0.1, 0.1), boundary, empty_slots=3)
    p = Params(core_a=1e-8, alpha=0.098, alpha_p=0.016, use_mf=1, dl_max=1e-2, use_bh=use_bh,
               bh_theta=0.5, vn=Flow("simple", {"external_v": (0.5, 0, 0)}))
    a = oracle.update_tangle(t, p, 0.0)
    b = ref.update_tangle(t, p, 0.0)
    assert rel_err(a.vels, b.vels, t.active) < TOL_V
    assert pos_err(oracle.rk4_step(a, p, 0.0, 1e-6).pos, ref.rk4_step(b, p, 0.0, 1e-6).pos, t.active) < 1e-14
