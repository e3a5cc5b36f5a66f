"""Golden-fixture loading shared by the tests."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

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
