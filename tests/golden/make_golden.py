"""Generate the golden fixtures in tests/golden/*.npz from the UNMODIFIED
OpenVort reference (oracle/_ref/libov_ref.so, compiled from the reference's
own sources by oracle/Makefile).

    python tests/golden/make_golden.py

Each fixture in tests/golden/*.npz holds a seeded input tangle (positions,
links, status, box, boundary name), the run-time parameters, and the
reference's outputs:
dxi, tangents, normals, vels, vs after update_tangle, and for the RK4 cases
the positions after a number of rk4_step calls (update_tangle before each,
as the reference's main loop does, src/main.c:112-114).  flows16.npz runs
every flow of the reference's table; samples/cfg2_bh4.npz holds the
reference's velocities at sample nodes of a tangle the tests regenerate
from its seed.

    python tests/golden/make_golden.py [fixture ...]
"""
from __future__ import annotations

import dataclasses
import json
import sys
from dataclasses import asdict
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from openvort_b200 import geometry as G  # noqa: E402
from openvort_b200.tangle import Flow, Params  # noqa: E402
from oracle.oracle import Ref, build  # noqa: E402

sys.path.insert(0, str(ROOT / "tests"))
from cases import CFG2, CFG2_SEED_SAMPLES, CFG2_SEEDS, cfg2_params, cfg2_sample_name, cfg2_tangle  # noqa: E402

OUT = Path(__file__).resolve().parent


def params_json(p: Params) -> str:
    d = asdict(p)
    return json.dumps(d)


def cases():
    ring_p = Params(core_a=1.3e-8, use_mf=0, alpha=0.0, alpha_p=0.0, hyperfriction=0,
                    dl_max=2 * 2 * np.pi * 1e-2 / 256)
    yield "ring256", G.single_ring(256, 1e-2), ring_p, {"rk4_steps": 10, "dt": 5e-6}
    per_p = Params(core_a=1.3e-8, alpha=0.098, alpha_p=0.016, dl_max=2 * 0.1 / 200,
                   vn=Flow("simple", {"external_v": (0.5, 0.0, 0.0)}))
    t = G.random_ring_tangle(1, 20, 0.1, boundary="periodic-26")
    yield "periodic26_direct", t, per_p, {"rk4_steps": 2, "dt": 1e-6}
    for th in (0.3, 0.4, 0.5):
        p = dataclasses.replace(per_p, use_bh=1, bh_theta=th)
        yield f"periodic26_bh{int(th * 10)}", t, p, {"rk4_steps": 1 if th == 0.4 else 0, "dt": 1e-6}
    # open boundaries, EMPTY holes between the nodes, hyperfriction on
    t2 = G.random_ring_tangle(2, 8, 0.1, boundary="open", empty_slots=17)
    t2.box_lo, t2.box_hi = (-0.05,) * 3, (0.15,) * 3
    t2._bind()
    p2 = Params(core_a=1.3e-8, alpha=0.1, alpha_p=0.01, dl_max=1e-3, hyperfriction=1,
                max_curv_scale=0.2, vn=Flow("simple", {"external_v": (0.0, 0.3, 0.0)}),
                vs=Flow("simple", {"external_v": (0.01, 0.0, 0.0)}))
    yield "open_empty_direct", t2, p2, {"rk4_steps": 1, "dt": 1e-6}
    yield "open_empty_bh4", t2, dataclasses.replace(p2, use_bh=1, bh_theta=0.4), {"rk4_steps": 0, "dt": 0}
    # a half ring pinned on a mirror wall: pinned stencils, mirror image, v_b
    w = G.wall_half_ring(64)
    pw = Params(core_a=1.3e-8, dl_max=2e-3, hyperfriction=0, alpha=0.05, alpha_p=0.01,
                vn=Flow("coscos", {"k": 50.0, "v0": 0.1, "l": 0.05}),
                vb=Flow("no flow"))
    yield "wall_half_ring", w, pw, {"rk4_steps": 0, "dt": 0}
    # periodic-z image table with a time-dependent flow
    t3 = G.random_ring_tangle(4, 6, 0.1, boundary="periodic-z-open-xy")
    p3 = Params(core_a=1e-8, alpha=0.1, alpha_p=0.02, dl_max=1e-3,
                vn=Flow("oscillating", {"strength": 0.3, "frequency": 50.0,
                                        "wave": (10.0, 0.0, 5.0), "polarization": (0.0, 1.0, 0.0)}),
                vs=Flow("rotosc", {"freq": 20.0, "amp": 0.5}))
    yield "periodic_z_flows", t3, p3, {"rk4_steps": 1, "dt": 1e-6, "time": 0.003}


# Every flow of the reference's table (src/external_velocity.c:85-174) with
# parameters that make it non-trivial on the flows tangle (centres in
# [0, 0.1]^3, evaluated at t = 3 ms).  "spherical and simple" is absent: the
# reference's function returns before writing its output (get_v_simple
# returns 1, read as an error at :235-237), so update_velocity adds an
# uninitialised stack value; tests/test_oracle.py pins that behaviour and the
# GPU's sum of the two flows is checked against the two recorded separately.
FLOWS16 = [
    ("no flow", {}),
    ("spherical", {"strength": 2e-3, "cutoff": 0.02}),
    ("simple", {"external_v": (0.3, -0.1, 0.2)}),
    ("cylindrical", {"strength": 2e-3, "cutoff": 0.02}),
    ("oscillating", {"strength": 0.3, "frequency": 50.0, "wave": (10.0, 3.0, 5.0),
                     "polarization": (0.2, 1.0, -0.4)}),
    ("oscillating slit", {"strength": 0.4, "frequency": 40.0, "cutoff": 0.03}),
    ("coscos", {"k": 50.0, "v0": 0.1, "l": 0.05}),
    ("coscos-divfree", {"k": 50.0, "v0": 0.1, "l": 0.05}),
    ("cos-divfree", {"k": 40.0, "v0": 0.2, "l": 0.07}),
    ("simple-shear", {"rate": 3.0, "v0": 0.1}),
    ("rotosc", {"freq": 20.0, "amp": 0.5}),
    ("DG", {"rot": 2.0, "vz": 0.1}),
    ("rotosc-boundary", {"freq": 30.0, "amp": 0.7}),
    ("constant acceleration", {"accel": 30.0}),
    ("parabolic", {"H": 0.1, "amp": 20.0}),
]
FLOWS_TIME = 0.003


def flows16(ref):
    """One tangle, each flow once as vn_conf (mutual friction) and once as
    vs_conf; the fixture's base arrays are the no-flow run."""
    t = G.random_ring_tangle(7, 5, 0.1, boundary="open")
    t.box_lo, t.box_hi = (-0.05,) * 3, (0.15,) * 3
    t._bind()
    base = Params(core_a=1e-8, alpha=0.1, alpha_p=0.02, dl_max=1e-3, hyperfriction=0,
                  vn=Flow("no flow"), vs=Flow("no flow"))
    u = ref.update_tangle(t, base, FLOWS_TIME)
    arrays = dict(pos=t.pos, fwd=t.links[:, 0], rev=t.links[:, 1], status=t.stat[:, 0],
                  pin_wall=t.stat[:, 1], box_lo=np.array(t.box_lo), box_hi=np.array(t.box_hi),
                  dxi=u.dxi, tangents=u.tangents, normals=u.normals, vels=u.vels, vs=u.vs)
    for i, (fname, prm) in enumerate(FLOWS16):
        for which in ("vn", "vs"):
            p = dataclasses.replace(base, **{which: Flow(fname, prm)})
            r = ref.update_tangle(t, p, FLOWS_TIME)
            arrays[f"vels_{which}_{i}"] = r.vels
            if which == "vs":       # vn_conf enters only vels
                arrays[f"vs_{which}_{i}"] = r.vs
    flows = [{"name": n, "params": {k: (list(v) if isinstance(v, tuple) else v) for k, v in prm.items()}}
             for n, prm in FLOWS16]
    meta = {"boundary": t.boundary, "params": json.loads(params_json(base)), "time": FLOWS_TIME,
            "rk4_steps": 0, "dt": 0, "flows": flows}
    np.savez_compressed(OUT / "flows16.npz", meta=np.array(json.dumps(meta)), **arrays)
    print("flows16", t.n, "nodes")


def cfg2_samples(ref, seed=None):
    """The 22.4k-point periodic tangle of the config-2 workload (regenerated
    by the tests from its seed; a checksum pins it): the reference's vs
    (update_velocity: local term, flow, Biot-Savart, 26 images) at seeded
    sample nodes with its octree at theta 0.4 and with its direct sum."""
    import ctypes as C
    t = cfg2_tangle(seed)
    rng = np.random.default_rng(CFG2["seed"] if seed is None else seed)
    size = CFG2["samples"] if seed is None else CFG2_SEED_SAMPLES
    idx = np.sort(rng.choice(np.nonzero(t.active)[0], size=size, replace=False)).astype(np.int32)
    out = {}
    for name, use_bh in (("vs_bh4", 1), ("vs_direct", 0)):
        p = cfg2_params(use_bh)
        ref.configure(p)
        tt = t.copy()
        tt.set_images_from_library(ref.lib)
        ref.lib.update_tangents_normals.restype = None
        ref.lib.update_tangents_normals(C.cast(tt.ptr(), C.c_void_p))
        f = ref.lib.refh_sample_vs
        f.restype = None
        f.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                      C.POINTER(C.c_double)]
        v = np.zeros((len(idx), 3))
        tb = C.c_double()
        f(C.cast(tt.ptr(), C.c_void_p), 0.0, idx.ctypes.data, len(idx), use_bh, v.ctypes.data, C.byref(tb))
        out[name] = v
    meta = {**CFG2, "seed": CFG2["seed"] if seed is None else seed, "samples": size, "n": t.n,
            "pos_sum": float(np.sum(t.pos)), "pos_abs_sum": float(np.sum(np.abs(t.pos)))}
    (OUT / "samples").mkdir(exist_ok=True)
    name = cfg2_sample_name(seed)
    np.savez_compressed(OUT / "samples" / (name + ".npz"), meta=np.array(json.dumps(meta)), idx=idx, **out)
    print(name, "samples", t.n, "nodes")


def main():
    build()
    ref = Ref(threads=8)
    only = sys.argv[1:]
    if not only or "flows16" in only:
        flows16(ref)
    if not only or "cfg2_bh4" in only:
        cfg2_samples(ref)
    for seed in CFG2_SEEDS:
        if not only or cfg2_sample_name(seed) in only:
            cfg2_samples(ref, seed)
    for name, t, p, opt in cases():
        if only and name not in only:
            continue
        time = opt.get("time", 0.0)
        u = ref.update_tangle(t, p, time)
        arrays = dict(pos=t.pos, fwd=t.links[:, 0], rev=t.links[:, 1], status=t.stat[:, 0],
                      pin_wall=t.stat[:, 1], box_lo=np.array(t.box_lo), box_hi=np.array(t.box_hi),
                      dxi=u.dxi, tangents=u.tangents, normals=u.normals, vels=u.vels, vs=u.vs)
        meta = {"boundary": t.boundary, "params": json.loads(params_json(p)), "time": time,
                "rk4_steps": opt["rk4_steps"], "dt": opt["dt"]}
        cur = u
        tt = time
        for s in range(opt["rk4_steps"]):
            nxt = ref.rk4_step(cur, p, tt, opt["dt"])
            tt += opt["dt"]
            cur = ref.update_tangle(nxt, p, tt)
            arrays[f"rk4_pos_{s + 1}"] = cur.pos
        np.savez_compressed(OUT / f"{name}.npz", meta=np.array(json.dumps(meta)), **arrays)
        print(name, t.n, "nodes")


if __name__ == "__main__":
    main()
