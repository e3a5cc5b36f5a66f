"""Golden-fixture loading shared by the tests."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from openvort_b200 import geometry as G
from openvort_b200.tangle import Flow, HostTangle, Params

GOLDEN = Path(__file__).resolve().parent / "golden"
NAMES = sorted(p.stem for p in GOLDEN.glob("*.npz"))


def params_from(d: dict) -> Params:
    d = dict(d)
    for k in ("vn", "vs", "vb"):
        f = d[k]
        params = {n: (tuple(v) if isinstance(v, list) else v) for n, v in f["params"].items()}
        d[k] = Flow(f["name"], params)
    return Params(**d)


def load(name: str, alloc=np.empty):
    z = np.load(GOLDEN / f"{name}.npz")
    meta = json.loads(str(z["meta"]))
    t = HostTangle(z["pos"], z["fwd"], z["rev"], z["status"], z["pin_wall"], tuple(z["box_lo"]),
                   tuple(z["box_hi"]), meta["boundary"], alloc=alloc)
    return t, params_from(meta["params"]), meta, z


def rel_err(a, b, mask=None) -> float:
    """max over nodes of |a - b| / |b|"""
    a = np.asarray(a)
    b = np.asarray(b)
    if mask is not None:
        a, b = a[mask], b[mask]
    if len(a) == 0:
        return 0.0
    num = np.linalg.norm(a - b, axis=-1)
    den = np.linalg.norm(b, axis=-1)
    den = np.where(den > 0, den, 1.0)
    return float(np.max(num / den))


def pos_err(a, b, mask=None) -> float:
    """max position difference relative to the largest coordinate extent"""
    a = np.asarray(a)
    b = np.asarray(b)
    if mask is not None:
        a, b = a[mask], b[mask]
    scale = max(1e-30, float(np.max(np.abs(b))))
    return float(np.max(np.abs(a - b))) / scale


def fixture_flows(meta: dict):
    """(index, Flow) of each flow recorded in a flows fixture."""
    return [(i, Flow(f["name"], {n: (tuple(v) if isinstance(v, list) else v) for n, v in f["params"].items()}))
            for i, f in enumerate(meta["flows"])]


# The config-2 workload's tangle (512 rings in a periodic cube D = 0.1 cm,
# radii U[0.02, 0.05] D, dl = D/200, 26 images: 22,379 points), rebuilt from
# its seed; samples/cfg2_bh4.npz holds the reference's velocities at seeded
# sample nodes of it and a checksum of its positions.
CFG2 = {"seed": 2026, "rings": 512, "D": 0.1, "dl": 0.1 / 200, "samples": 256}
# further seeds of the same workload (samples/cfg2_bh4_s<seed>.npz), fewer
# sample nodes each
CFG2_SEEDS = (0, 1, 2, 3, 4)
CFG2_SEED_SAMPLES = 64


def cfg2_params(use_bh: int) -> Params:
    return Params(core_a=1e-8, alpha=0.098, alpha_p=0.016, use_mf=1, dl_max=2 * CFG2["dl"],
                  hyperfriction=1, use_bh=use_bh, bh_theta=0.4, bh_grain=1e-8,
                  vn=Flow("simple", {"external_v": (0.5, 0.0, 0.0)}), vs=Flow("no flow"))


def cfg2_tangle(seed: int | None = None):
    seed = CFG2["seed"] if seed is None else seed
    return G.random_ring_tangle(seed, CFG2["rings"], CFG2["D"], dl=CFG2["dl"], boundary="periodic-26")


def cfg2_sample_name(seed: int | None = None) -> str:
    return "cfg2_bh4" if seed is None else f"cfg2_bh4_s{seed}"


def load_cfg2_samples(seed: int | None = None):
    """(tangle, sample fixture); asserts the regenerated tangle is the one
    the reference ran on."""
    z = np.load(GOLDEN / "samples" / (cfg2_sample_name(seed) + ".npz"))
    meta = json.loads(str(z["meta"]))
    t = cfg2_tangle(seed)
    assert t.n == meta["n"] and float(np.sum(t.pos)) == meta["pos_sum"] and \
        float(np.sum(np.abs(t.pos))) == meta["pos_abs_sum"], "generator no longer reproduces the tangle"
    return t, z
