"""GPU parity: libov_gpu.so, called through its C ABI (the reference-named
entry points and ov_state_*), against the reference's golden fixtures and the
CPU oracle on the same seeded inputs.

Tolerances (max over nodes of |dv| / |v_ref|):
  FP64 path   1e-12 on velocities (tangents 1e-11, normals 1e-10: second
              differences of positions ~dl apart lose ~3 digits, and the
              stencil weights are factored differently from the reference)
  mixed path  1e-5 on velocities
"""
import ctypes as C
import dataclasses

import numpy as np
import pytest

from cases import NAMES, fixture_flows, load, pos_err, rel_err
from openvort_b200 import geometry as G
from openvort_b200.tangle import Flow, Params, Vec3d
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

TOL_V64, TOL_T64, TOL_N64, TOL_MIXED = 1e-12, 1e-11, 1e-10, 1e-5


@pytest.fixture(scope="module")
def ov():
    import openvort_b200 as ov
    lib = ov.load()
    assert lib.ov_init(0) == 0, lib.ov_last_error_message()
    return ov


@pytest.fixture(scope="module")
def oracle():
    return Oracle()


def gpu_update(ov, t, p, time=0.0, precision=0):
    ov.configure(p, precision)
    out = t.copy()
    ov.update_tangle(out, time)
    return out


@pytest.mark.parametrize("name", NAMES)
def test_update_tangle_fp64_vs_golden(ov, name):
    t, p, meta, z = load(name)
    out = gpu_update(ov, t, p, meta["time"])
    act = t.active
    assert np.max(np.abs(out.dxi - z["dxi"])[act]) <= 1e-15 * np.max(z["dxi"][act])
    assert rel_err(out.tangents, z["tangents"], act) < TOL_T64
    assert rel_err(out.normals, z["normals"], act) < TOL_N64
    assert rel_err(out.vs, z["vs"], act) < TOL_V64
    assert rel_err(out.vels, z["vels"], act) < TOL_V64


@pytest.mark.parametrize("name", NAMES)
def test_update_tangle_mixed_vs_golden(ov, name):
    t, p, meta, z = load(name)
    out = gpu_update(ov, t, p, meta["time"], precision=1)
    assert rel_err(out.vels, z["vels"], t.active) < TOL_MIXED


@pytest.mark.parametrize("name", [n for n in NAMES if n in ("ring256", "periodic26_direct",
                                                           "periodic26_bh4", "open_empty_direct",
                                                           "periodic_z_flows")])
def test_rk4_fp64_vs_golden(ov, name):
    t, p, meta, z = load(name)
    ov.configure(p, 0)
    cur = t.copy()
    tt = meta["time"]
    ov.update_tangle(cur, tt)
    for s in range(meta["rk4_steps"]):
        ov.rk4_step(cur, tt, meta["dt"])
        tt += meta["dt"]
        ov.update_tangle(cur, tt)
        assert pos_err(cur.pos, z[f"rk4_pos_{s + 1}"], t.active) < 1e-14


@pytest.mark.parametrize("which", ["vn", "vs"])
def test_all_external_flows_fp64_vs_reference(ov, which):
    """Each flow of the reference's table (src/external_velocity.c:85-174)
    as vn_conf (through mutual friction) and as vs_conf, FP64, against the
    reference's own update_tangle on the same tangle and time."""
    t, base, meta, z = load("flows16")
    act = t.active
    flows = fixture_flows(meta)
    assert len(flows) == 15
    for i, f in flows:
        out = gpu_update(ov, t, dataclasses.replace(base, **{which: f}), meta["time"])
        assert rel_err(out.vels, z[f"vels_{which}_{i}"], act) < TOL_V64, f.name
        want_vs = z[f"vs_vs_{i}"] if which == "vs" else z["vs"]
        assert rel_err(out.vs, want_vs, act) < TOL_V64, f.name


@pytest.mark.parametrize("which", ["vn", "vs"])
def test_spherical_and_simple_is_the_sum_of_its_parts(ov, which):
    """The reference's "spherical and simple" returns before writing its
    output (src/external_velocity.c:226-237), so its own result is an
    uninitialised value.  The library gives spherical + simple: since vs and
    vels are affine in the external flow, that equals the reference's
    spherical run plus its simple run minus its no-flow run."""
    t, base, meta, z = load("flows16")
    act = t.active
    idx = {f.name: (i, f) for i, f in fixture_flows(meta)}
    (i_sph, sph), (i_sim, sim), (i_0, _) = idx["spherical"], idx["simple"], idx["no flow"]
    assert sph.params["cutoff"] > 0
    both = Flow("spherical and simple", {**sph.params, **sim.params})
    out = gpu_update(ov, t, dataclasses.replace(base, **{which: both}), meta["time"])
    want = z[f"vels_{which}_{i_sph}"] + z[f"vels_{which}_{i_sim}"] - z[f"vels_{which}_{i_0}"]
    assert rel_err(out.vels, want, act) < TOL_V64


def test_config2_tangle_bh4_and_direct_vs_reference(ov):
    """The 22.4k-point periodic tangle of the config-2 workload: FP64
    Barnes-Hut (theta 0.4) and direct sums against the reference's
    update_velocity at 256 sample nodes, and the mixed form within its
    tolerance of the same."""
    from cases import cfg2_params, load_cfg2_samples
    t, z = load_cfg2_samples()
    idx = z["idx"]
    for use_bh, key in ((1, "vs_bh4"), (0, "vs_direct")):
        out = gpu_update(ov, t, cfg2_params(use_bh))
        assert rel_err(out.vs[idx], z[key]) < TOL_V64, key
        mixed = gpu_update(ov, t, cfg2_params(use_bh), precision=1)
        assert rel_err(mixed.vs[idx], z[key]) < TOL_MIXED, key


@pytest.mark.parametrize("seed", [0, 1, 2, 3, 4])
def test_config2_seeds_bh4_and_direct_vs_reference(ov, seed):
    """Config 2's seeds 0..4 (22.5k-22.8k points each): FP64 Barnes-Hut
    (theta 0.4) and direct sums against the reference's update_velocity at
    64 sample nodes per tangle, and the mixed form within its tolerance."""
    from cases import cfg2_params, load_cfg2_samples
    t, z = load_cfg2_samples(seed)
    idx = z["idx"]
    for use_bh, key in ((1, "vs_bh4"), (0, "vs_direct")):
        out = gpu_update(ov, t, cfg2_params(use_bh))
        assert rel_err(out.vs[idx], z[key]) < TOL_V64, key
        mixed = gpu_update(ov, t, cfg2_params(use_bh), precision=1)
        assert rel_err(mixed.vs[idx], z[key]) < TOL_MIXED, key


def test_refined_fp64_reciprocals_match_ieee(ov):
    """The direct sum's FP64 1/sqrt(x) and 1/x (hardware approximation plus
    two Newton-Raphson steps) stay within 4 ulps of IEEE sqrt and division
    over 2^-128 .. 2^128."""
    lib = ov.load()
    a, b = C.c_double(-1), C.c_double(-1)
    assert lib.ov_check_fast_math(C.byref(a), C.byref(b)) == 0, lib.ov_last_error_message()
    assert 0 <= a.value <= 4.0 and 0 <= b.value <= 4.0, (a.value, b.value)


def test_device_state_run_vs_oracle(ov, oracle):
    """ov_state_run (device-resident update_tangle + rk4_step) against the
    oracle stepping the same tangle on the CPU."""
    t, p, meta, z = load("periodic26_bh4")
    ov.configure(p, 0)
    st = ov.DeviceState(t.copy())
    st.run(0.0, 1e-6, 3)
    st.download()
    cur = oracle.update_tangle(t, p, 0.0)
    tt = 0.0
    for _ in range(3):
        nxt = oracle.rk4_step(cur, p, tt, 1e-6)
        tt += 1e-6
        cur = oracle.update_tangle(nxt, p, tt)
    assert pos_err(st.t.pos, cur.pos, t.active) < 1e-14
    st.close()


@pytest.mark.parametrize("theta", [0.3, 0.5])
def test_bh_larger_tangle_vs_oracle(ov, oracle, theta):
    """~4k nodes, periodic-26, both precisions against the FP64 oracle."""
    t = G.random_ring_tangle(3, 100, 0.1, boundary="periodic-26", empty_slots=9)
    p = Params(core_a=1.3e-8, alpha=0.098, alpha_p=0.016, dl_max=1e-3, use_bh=1, bh_theta=theta,
               vn=Flow("simple", {"external_v": (0.5, 0, 0)}))
    ref = oracle.update_tangle(t, p)
    g64 = gpu_update(ov, t, p)
    assert rel_err(g64.vels, ref.vels, t.active) < TOL_V64
    gmx = gpu_update(ov, t, p, precision=1)
    assert rel_err(gmx.vels, ref.vels, t.active) < TOL_MIXED


@pytest.mark.parametrize("boundary,seed", [("periodic-26", 5), ("open", 6)])
def test_nodes_outside_the_root_box_vs_oracle(ov, oracle, boundary, seed):
    """Nodes pushed just outside the root box (as RK4 steps without
    enforce_boundaries leave them) drop out of every subtree but count in the
    root's moments (src/vec3_maths.c:67-77, src/octree.c:118-127); the walk
    gives each its own warp at the front of its target list.  Both
    precisions against the FP64 oracle, with and without them."""
    # (open seed 5 has a node whose sum the summation order moves by 2e-13
    # even between the oracle and the reference; seed 6 has none)
    t = G.random_ring_tangle(seed, 100, 0.1, boundary=boundary, empty_slots=5)
    lo = np.array(t.struct.box.bottom_left_back.p[:])
    hi = np.array(t.struct.box.top_right_front.p[:])
    a = np.nonzero(t.active)[0]
    # the nodes nearest each face, moved 1e-6 cm past it
    moved = []
    for ax in range(3):
        for side, lim in ((0, lo[ax]), (1, hi[ax])):
            d = np.abs(t.pos[a, ax] - lim)
            for k in a[np.argsort(d)[:3]]:
                if k in moved:
                    continue
                t.pos[k, ax] = lim - 1e-6 if side == 0 else lim + 1e-6
                moved.append(k)
    assert len(moved) >= 12
    p = Params(core_a=1.3e-8, alpha=0.098, alpha_p=0.016, dl_max=1e-3, use_bh=1, bh_theta=0.5,
               vn=Flow("simple", {"external_v": (0.5, 0, 0)}))
    ref = oracle.update_tangle(t, p)
    assert rel_err(gpu_update(ov, t, p).vels, ref.vels, t.active) < TOL_V64
    assert rel_err(gpu_update(ov, t, p, precision=1).vels, ref.vels, t.active) < TOL_MIXED


def test_quadtree_vs_oracle(ov, oracle):
    t = G.random_ring_tangle(8, 30, 0.1, boundary="periodic-6")
    p = Params(core_a=1.3e-8, alpha=0.1, alpha_p=0.01, dl_max=1e-3, use_bh=1, bh_theta=0.4,
               bh_quadtree=1)
    assert rel_err(gpu_update(ov, t, p).vels, oracle.update_tangle(t, p).vels, t.active) < TOL_V64


def test_point_queries(ov, oracle):
    """calculate_vs / calculate_vs_shift / octree_get_vs at arbitrary points."""
    t, p, _, _ = load("periodic26_bh4")
    lib = ov.load()
    ov.configure(p, 0)
    t.set_images_from_library(lib)
    rng = np.random.default_rng(7)
    pts = rng.uniform(0, 0.1, size=(8, 3))
    skip = [-1, 3, 10, -1, 50, 7, -1, 0]
    want = oracle.segments_at(t, p, pts, np.array(skip, np.int32))
    for i in range(8):
        v = lib.calculate_vs(t.ptr(), Vec3d((C.c_double * 3)(*pts[i])), skip[i])
        ov.check(lib)
        assert rel_err(np.array(v.p)[None], want[i:i + 1]) < TOL_V64
    # calculate_vs_shift with a node list and a shift
    only = np.arange(0, t.n, 3, dtype=np.int32)
    sh = Vec3d((C.c_double * 3)(0.01, -0.02, 0.005))
    v = lib.calculate_vs_shift(t.ptr(), Vec3d((C.c_double * 3)(*pts[0])), -1, C.byref(sh),
                               only.ctypes.data_as(C.POINTER(C.c_int)), len(only))
    ov.check(lib)
    sub = t.copy()
    sub.links[np.setdiff1d(np.arange(t.n), only), 0] = -1
    w = oracle.segments_at(sub, p, pts[:1] + np.array([0.01, -0.02, 0.005]))
    assert rel_err(np.array(v.p)[None], w) < TOL_V64
    # octree_build / octree_get_vs (no images), at the build theta and another
    tree = lib.octree_build(t.ptr(), 0)
    ov.check(lib)
    want = oracle.bh_at(t, p, pts, np.array(skip, np.int32))
    for i in range(8):
        res = Vec3d()
        lib.octree_get_vs(tree, C.byref(Vec3d((C.c_double * 3)(*pts[i]))), p.bh_theta, C.byref(res), skip[i])
        ov.check(lib)
        assert rel_err(np.array(res.p)[None], want[i:i + 1]) < TOL_V64
    p2 = dataclasses.replace(p, bh_theta=0.25)
    want2 = oracle.bh_at(t, p2, pts[:2])
    for i in range(2):
        res = Vec3d()
        lib.octree_get_vs(tree, C.byref(Vec3d((C.c_double * 3)(*pts[i]))), 0.25, C.byref(res), -1)
        assert rel_err(np.array(res.p)[None], want2[i:i + 1]) < TOL_V64
    lib.octree_destroy(tree)


def test_update_velocity_single_node(ov):
    """update_velocity(k) (the reference's reconnection calls it per node)
    equals node k of update_velocities, direct and with a tree."""
    for name in ("periodic26_direct", "periodic26_bh4"):
        t, p, meta, z = load(name)
        lib = ov.load()
        ov.configure(p, 0)
        cur = t.copy()
        cur.tangents[:] = z["tangents"]
        cur.normals[:] = z["normals"]
        cur.set_images_from_library(lib)
        tree = lib.octree_build(cur.ptr(), 0) if p.use_bh else None
        for k in (0, 17, 400, t.n - 1):
            cur.vels[k] = 0
            lib.update_velocity(cur.ptr(), k, 0.0, tree)
            ov.check(lib)
            assert rel_err(cur.vels[k:k + 1], z["vels"][k:k + 1]) < TOL_V64
        if tree:
            lib.octree_destroy(tree)


def test_update_velocities_with_user_tree(ov):
    t, p, meta, z = load("periodic26_bh3")
    lib = ov.load()
    ov.configure(p, 0)
    cur = t.copy()
    cur.tangents[:] = z["tangents"]
    cur.normals[:] = z["normals"]
    cur.set_images_from_library(lib)
    tree = lib.octree_build(cur.ptr(), 0)
    lib.update_velocities(cur.ptr(), 0.0, tree)
    ov.check(lib)
    lib.octree_destroy(tree)
    assert rel_err(cur.vels, z["vels"], t.active) < TOL_V64


def test_eval_points_direct_and_bh(ov, oracle):
    """ov_state_eval_points: direct and Barnes-Hut sums with the 26 images at
    arbitrary points, against the oracle summing the tangle and each image
    point the same way (src/tangle.c:611-638)."""
    t, p, _, _ = load("periodic26_bh5")
    ov.configure(p, 0)
    st = ov.DeviceState(t.copy())
    rng = np.random.default_rng(9)
    pts = rng.uniform(0, 0.1, size=(100, 3))
    from openvort_b200.tangle import IMAGE_TABLES
    L = 0.1
    ref_d = oracle.segments_at(t, p, pts)
    ref_b = oracle.bh_at(t, p, pts)
    for sh, _ in IMAGE_TABLES["periodic-26"]:
        ref_d = ref_d + oracle.segments_at(t, p, pts - L * np.array(sh))
        ref_b = ref_b + oracle.bh_at(t, p, pts - L * np.array(sh))
    assert rel_err(st.eval_points(pts, method=0), ref_d) < TOL_V64
    assert rel_err(st.eval_points(pts, method=1), ref_b) < TOL_V64
    st.close()


def test_ring_speed_thin_core_gpu(ov, oracle):
    """1000 RK4 steps of the 256-point ring (dt 5e-6): mean speed within 3 %
    of kappa/(4 pi R)(ln(8R/a) - 1/2) and equal to the oracle's first step."""
    R, a, kappa = 1e-2, 1.3e-8, 9.97e-4
    t = G.single_ring(256, R)
    p = Params(core_a=a, use_mf=0, alpha=0, alpha_p=0, hyperfriction=0, dl_max=2 * 2 * np.pi * R / 256)
    ov.configure(p, 0)
    st = ov.DeviceState(t.copy())
    z0 = t.pos[:, 2].mean()
    st.run(0.0, 5e-6, 1000)
    st.download()
    v = (st.t.pos[:, 2].mean() - z0) / (1000 * 5e-6)
    v_thin = kappa / (4 * np.pi * R) * (np.log(8 * R / a) - 0.5)
    assert abs(v / v_thin - 1) < 0.03
    # radius conserved to the discretisation
    c = st.t.pos.mean(axis=0)
    rr = np.linalg.norm(st.t.pos - c, axis=1)
    assert np.max(np.abs(rr / R - 1)) < 1e-3
    st.close()


def test_broken_links_fail_loudly(ov, monkeypatch):
    monkeypatch.setenv("OV_QUIET", "1")
    t = G.single_ring(32, 1e-2)
    t.links[5, 0] = -1   # a FREE node with no forward neighbour
    ov.configure(Params(use_mf=0, hyperfriction=0), 0)
    with pytest.raises(ov.OVError) as e:
        ov.update_tangents_normals(t)
    assert e.value.code == 3


def test_unknown_flow_fails_loudly(ov, monkeypatch):
    monkeypatch.setenv("OV_QUIET", "1")
    t = G.single_ring(32, 1e-2)
    p = Params(use_mf=1, hyperfriction=0, vn=Flow("simple", {"external_v": (1, 0, 0)}))
    lib = ov.configure(p, 0)
    conf, keep = Flow("simple", {"external_v": (1, 0, 0)}).vconf()
    conf.name = b"no such flow"
    C.memmove(C.addressof(type(conf).in_dll(lib, "vn_conf")), C.addressof(conf), C.sizeof(conf))
    with pytest.raises(ov.OVError) as e:
        ov.update_tangle(t, 0.0)
    assert e.value.code == 5


def test_mixed_vs_fp64_large_bh(ov):
    """Size-independent property at ~200k nodes: the mixed form stays within
    1e-5 of the FP64 form on the same tree and theta."""
    t = G.random_ring_tangle(21, G.rings_for_points(200_000, 0.2, dl=0.2 / 400), 0.2,
                             dl=0.2 / 400, boundary="periodic-26")
    p = Params(core_a=1.3e-8, alpha=0.098, alpha_p=0.016, dl_max=2 * 0.2 / 400, use_bh=1,
               bh_theta=0.5, vn=Flow("simple", {"external_v": (0.5, 0, 0)}))
    a = gpu_update(ov, t, p, precision=0)
    b = gpu_update(ov, t, p, precision=1)
    assert rel_err(b.vels, a.vels, t.active) < TOL_MIXED


def test_bh_tree_beyond_one_million_nodes(ov, oracle):
    """A tree of ~1.09M nodes: the preorder scan over the cells spans more
    than 1024 blocks of 1024 (its block sums are scanned in two rounds with a
    carry) and the root cell's moments are summed in 64 chunks.  FP64
    Barnes-Hut velocities at 48 points with the 26 periodic images, against
    the oracle's recursive tree."""
    from openvort_b200.tangle import IMAGE_TABLES
    D, dl = 0.4, 0.4 / 800
    t = G.random_ring_tangle(5, G.rings_for_points(1_100_000, D, dl=dl), D, dl=dl,
                             boundary="periodic-26")
    assert t.n > 1024 * 1024
    p = Params(core_a=1e-8, dl_max=2 * dl, use_bh=1, bh_theta=0.5, bh_grain=1e-8)
    ov.configure(p, 0)
    st = ov.DeviceState(t.copy())
    pts = np.random.default_rng(11).uniform(0, D, size=(48, 3))
    shifts = [(0, 0, 0)] + [sh for sh, _ in IMAGE_TABLES["periodic-26"]]
    allp = np.concatenate([pts - D * np.array(sh) for sh in shifts])
    ref = oracle.bh_at(t, p, allp).reshape(len(shifts), len(pts), 3).sum(axis=0)
    assert rel_err(st.eval_points(pts, method=1), ref) < TOL_V64
    st.close()


def _ring5():
    from openvort_b200.tangle import ring_points
    r = ring_points(np.array([0.05, 0.05, 0.05]), (0.3, 0.2, 0.9), 0.004, 5)
    return G.rings_to_tangle([r], (0, 0, 0), (0.1, 0.1, 0.1), "periodic-26", empty_slots=3)


@pytest.mark.parametrize("use_bh", [0, 1])
def test_smallest_loop_vs_oracle(ov, oracle, use_bh):
    """A 5-node loop among EMPTY slots: the tree has a handful of cells and
    every stencil reaches round the whole loop.  Velocities and one RK4 step
    in FP64 against the oracle; the mixed form within its tolerance."""
    t = _ring5()
    p = Params(core_a=1e-8, alpha=0.098, alpha_p=0.016, use_mf=1, dl_max=1e-2, use_bh=use_bh,
               bh_theta=0.5, vn=Flow("simple", {"external_v": (0.5, 0, 0)}))
    ref = oracle.update_tangle(t, p)
    g = gpu_update(ov, t, p)
    assert rel_err(g.vels, ref.vels, t.active) < TOL_V64
    ov.rk4_step(g, 0.0, 1e-6)
    assert pos_err(g.pos, oracle.rk4_step(ref, p, 0.0, 1e-6).pos, t.active) < 1e-14
    assert rel_err(gpu_update(ov, t, p, precision=1).vels, ref.vels, t.active) < TOL_MIXED


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("use_bh", [0, 1])
def test_tangles_without_nodes(ov, use_bh, precision):
    """N = 0, and slots that are all EMPTY: update_tangle, rk4_step and a
    device-resident run have nothing to do and report no error."""
    from openvort_b200.tangle import HostTangle
    p = Params(core_a=1e-8, use_bh=use_bh, bh_theta=0.5)
    for n in (0, 4):
        t = HostTangle(np.zeros((n, 3)), -np.ones(n, np.int32), -np.ones(n, np.int32),
                       np.full(n, -1, np.int32), -np.ones(n, np.int32), (0, 0, 0), (0.1, 0.1, 0.1),
                       "periodic-26")
        g = gpu_update(ov, t, p, precision=precision)
        ov.rk4_step(g, 0.0, 1e-6)
        assert np.array_equal(g.pos, t.pos)
        st = ov.DeviceState(t.copy())
        st.run(0.0, 1e-6, 2)
        st.download()
        assert np.array_equal(st.t.pos, t.pos)
        st.close()
