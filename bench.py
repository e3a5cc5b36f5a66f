#!/usr/bin/env python
"""Benchmark: OpenVort's velocity + RK4 path on the large periodic tangle.

Workload (one "step" = one RK4 step = 4 velocity evaluations: k1 by
update_tangle, then three stages, each with its own octree build):
  ~1M points: rings with centres uniform in a periodic cube D = 0.4 cm,
  orientations uniform on the sphere, radii uniform in [0.02, 0.05] D,
  spacing dl = D/800; 26 nearest periodic images; Barnes-Hut theta = 0.5;
  counterflow v_n = 0.5 cm/s along x, alpha = 0.098, alpha' = 0.016;
  dt = 1e-6 s; mixed precision (FP32 far field, FP64 positions / local term /
  near segments).  Seeded synthetic data.

Printed JSON line (rank 0): value = point-velocity evaluations per second
over all GPUs (N points x 4 evaluations per step / device time), plus RK4
steps/s, the plain FP64 form's rate, the mixed-vs-FP64 error, the error
against an FP64 direct sum on 4096 sample nodes, the roofline of the
Barnes-Hut walk kernel, the reference's CPU baseline, the end-to-end rate
through the reference-named C ABI with pinned host buffers, launches and
clocks.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "point-velocity evals/s & RK4 steps/s at 1M pts: mixed vs FP64, ≤1e-5 rel err"
UNIT = "point-velocity evals/s"
D = 0.4
DL = D / 800
FLOPS_P2P = 43.0   # per segment-point interaction (direct sum / tree leaves)


def _hbm_peak():
    """Measured copy bandwidth of this GPU model (GB/s), else 6650 (fallback)."""
    try:
        return float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


HBM_PEAK, HBM_PEAK_SOURCE = _hbm_peak()
FLOPS_CELL = 60.0  # per multipole evaluation (monopole + second-order terms + opening test)
# dram__bytes_read.sum + dram__bytes_write.sum of one mixed walk launch per
# point: 52.8 MB over 198,002 points in the ncu capture of this kernel on
# this generator (profiles/bh_walk_multi_mixed_200k.md), scaled by the points
WALK_DRAM_BYTES_PER_POINT = 267.0
WALK_TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of k_walk_multi<mixed> at "
                       "198,002 points (profiles/bh_walk_multi_mixed_200k.md), 267 B per point x points")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--points", type=int, default=1_000_000)
    ap.add_argument("--theta", type=float, default=0.5)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--dt", type=float, default=1e-6)
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the direct-sum and batch lines")
    ap.add_argument("--batch-steps", type=int, default=200)
    ap.add_argument("--batch-systems", type=int, default=4096)
    ap.add_argument("--cfg1-steps", type=int, default=1000)
    ap.add_argument("--cfg2-steps", type=int, default=500)
    ap.add_argument("--cfg2-direct-steps", type=int, default=20)
    ap.add_argument("--adjoint-steps", type=int, default=2000)
    ap.add_argument("--shard", action="store_true",
                    help="at one GPU too: the sharded one-tangle run (the default when --gpus > 1)")
    ap.add_argument("--only", choices=["walk", "walk64", "direct", "batch", "cfg2", "adjoint", "reconnect"],
                    help="run one part alone and print its object (for profiling)")
    ap.add_argument("--independent", action="store_true",
                    help="with --gpus > 1: one independent tangle per rank (weak scaling) as the headline")
    return ap.parse_args()


def params(theta):
    from openvort_b200.tangle import Flow, Params
    return Params(core_a=1e-8, alpha=0.098, alpha_p=0.016, use_mf=1, dl_max=2 * DL, hyperfriction=1,
                  max_curv_scale=0.2, hyperalpha=0.5, use_bh=1, bh_theta=theta, bh_grain=1e-8,
                  vn=Flow("simple", {"external_v": (0.5, 0.0, 0.0)}), vs=Flow("no flow"))


def make_tangle(points, seed, alloc=np.empty, empty_slots=0):
    from openvort_b200 import geometry as G
    n_rings = G.rings_for_points(points, D, dl=DL)
    return G.random_ring_tangle(seed, n_rings, D, dl=DL, boundary="periodic-26", alloc=alloc,
                                empty_slots=empty_slots), n_rings


def pinned_alloc():
    import torch

    keep = []

    def alloc(shape, dtype):
        tdt = {np.dtype(np.float64): torch.float64, np.dtype(np.int32): torch.int32}[np.dtype(dtype)]
        t = torch.empty(shape, dtype=tdt, pin_memory=True)
        keep.append(t)
        return t.numpy()

    return alloc, keep


class Clocks:
    """nvidia-smi samples during the timed region (every 200 ms)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        rows = []
        for line in Path(self.f.name).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(args):
    from openvort_b200 import dist as D
    # a rank waits at most for rank 0's accuracy checks (tens of seconds):
    # a stuck peer ends the next collective with an error well before this
    r = D.setup(timeout_s=180.0)
    if r.world == 1:
        import torch
        if torch.cuda.is_available():
            r.device = f"cuda:{r.local}"
    return r.world, r.rank, r.local, r


def max_over_ranks(r, x: float) -> float:
    from openvort_b200 import dist as D
    return D.max_over_ranks(r, x)


def barrier(r):
    from openvort_b200 import dist as D
    D.barrier(r)


# ---------------------------------------------------------------- CPU side
def cpu_reference_sample(tangle, p, target_s=10.0, time0=0.0):
    """The reference's own per-evaluation work (update_tangents_normals,
    octree_build, update_velocity on a seeded sample of nodes, OpenMP over all
    host cores) from oracle/_ref; returns point-evals/s extrapolated to the
    whole tangle and a description."""
    from oracle.oracle import Ref, have_ref
    if not have_ref():
        return None
    threads = os.cpu_count() or 1
    ref = Ref(threads=threads)
    ref.configure(p)
    t = tangle.copy()
    t.set_images_from_library(ref.lib)
    f = ref.lib.refh_sample_eval
    f.restype = None
    f.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_int, C.POINTER(C.c_double),
                  C.POINTER(C.c_double), C.POINTER(C.c_double)]
    rng = np.random.default_rng(7)
    act = np.nonzero(t.active)[0]
    tg, tb, tn = C.c_double(), C.c_double(), C.c_double()
    # probe with a few nodes, then size the sample for ~target_s of node work
    m = 64
    idx = np.ascontiguousarray(rng.choice(act, size=m, replace=False).astype(np.int32))
    f(C.cast(t.ptr(), C.c_void_p), time0, idx.ctypes.data, m, C.byref(tg), C.byref(tb), C.byref(tn))
    per = max(tn.value / m, 1e-7)
    m = int(min(len(act), max(64, target_s / per)))
    idx = np.ascontiguousarray(rng.choice(act, size=m, replace=False).astype(np.int32))
    f(C.cast(t.ptr(), C.c_void_p), time0, idx.ctypes.data, m, C.byref(tg), C.byref(tb), C.byref(tn))
    n = len(act)
    t_eval = tg.value + tb.value + tn.value * n / m
    return {"value": n / t_eval, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": (f"reference update_tangents_normals + octree_build on all {n} nodes "
                       f"({tg.value:.2f} s + {tb.value:.2f} s) and update_velocity on {m} seeded nodes "
                       f"({tn.value:.2f} s, OpenMP {threads} threads), extrapolated to one evaluation "
                       f"of all nodes: {t_eval:.1f} s")}


def bench_config(args, n, n_job, n_rings, world) -> dict:
    """The workload description both arms print."""
    return {"workload": f"large periodic tangle: {n} points per GPU ({n_rings} rings, D=0.4 cm, "
                        f"dl=D/800, radii U[0.02,0.05]D), 26 periodic images, Barnes-Hut "
                        f"theta={args.theta}, mixed FP32/FP64, RK4 dt={args.dt}",
            "points": n, "points_all_ranks": n_job, "theta": args.theta, "images": 26,
            "dt": args.dt,
            "parallelism": f"{world} independent tangles (one per GPU)" if world > 1 else "1 GPU",
            "l2": "working set (octree cells + node table) larger than the 126 MB L2"}


def run_reference_arm(args, world, rank):
    p = params(args.theta)
    tangle, n_rings = make_tangle(args.points, args.seed)
    vals = []
    # warm-up samples are small; each timed step is one sampled evaluation
    for _ in range(args.warmup):
        cpu_reference_sample(tangle, p, target_s=0.5)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        r = cpu_reference_sample(tangle, p, target_s=8.0)
        if r is None:
            print(json.dumps({"impl": "reference",
                              "unavailable": "oracle/_ref/libov_ref.so (reference compiled from its sources) is not built"}))
            return
        vals.append(r)
    timed_s = time.perf_counter() - t0
    v = statistics.median([r["value"] for r in vals])
    n = int(tangle.active.sum())
    ms_step = 4 * n / v * 1e3
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(args, n, n, n_rings, world),
            "extrapolated": True,
            "timed_s": timed_s,
            "step_meaning": (f"each of the {args.steps} timed steps is one sampled evaluation (see "
                             "cpu_baseline.sample) extrapolated to all nodes; ms_per_step is the RK4 step "
                             "(4 evaluations) those samples imply, not wall time"),
            "rk4_steps_per_s": 1e3 / ms_step,
            "cpu_baseline": {**vals[-1], "value": v},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def dist_stats(e: np.ndarray) -> dict:
    return {"max": float(np.max(e)), "p99": float(np.percentile(e, 99)), "median": float(np.median(e))}


def bh_reference_check(tangle, p, idx, bh64, direct, vs64, n_direct=64):
    """The reference's own Barnes-Hut error on the sample nodes: its
    update_velocity (oracle/_ref) with its octree at all sample nodes, and
    with its direct sum at the first n_direct of them.  Reported beside the
    GPU's FP64 Barnes-Hut and direct sums at the same nodes, all relative to
    the direct-sum superfluid velocity."""
    from oracle.oracle import Ref, have_ref
    if not have_ref():
        return None
    ref = Ref(threads=os.cpu_count() or 1)
    ref.configure(p)
    t = tangle.copy()
    t.set_images_from_library(ref.lib)
    ref.lib.update_tangents_normals.restype = None
    ref.lib.update_tangents_normals(C.cast(t.ptr(), C.c_void_p))
    f = ref.lib.refh_sample_vs
    f.restype = None
    f.argtypes = [C.c_void_p, C.c_double, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.POINTER(C.c_double)]
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    m = len(idx)
    tb = C.c_double()
    t0 = time.perf_counter()
    ref_bh = np.zeros((m, 3))
    f(C.cast(t.ptr(), C.c_void_p), 0.0, idx.ctypes.data, m, 1, ref_bh.ctypes.data, C.byref(tb))
    t1 = time.perf_counter()
    t_build = tb.value
    nd = min(n_direct, m)
    ref_direct = np.zeros((nd, 3))
    f(C.cast(t.ptr(), C.c_void_p), 0.0, idx.ctypes.data, nd, 0, ref_direct.ctypes.data, C.byref(tb))
    t2 = time.perf_counter()
    # GPU superfluid velocities at the sample nodes: FP64 with the tree, and
    # with the direct sum in place of the tree's Biot-Savart sum
    gpu_bh = vs64[idx]
    gpu_direct = vs64[idx] - bh64 + direct
    norm = np.linalg.norm(gpu_direct, axis=1)

    def rel(a, b, k=None):
        k = len(a) if k is None else k
        return np.linalg.norm(a[:k] - b[:k], axis=1) / norm[:k]
    return {
        "nodes": m, "direct_nodes": nd,
        "reference_bh_vs_reference_direct": dist_stats(rel(ref_bh, ref_direct, nd)),
        "gpu_bh_fp64_vs_gpu_direct_same_nodes": dist_stats(rel(gpu_bh, gpu_direct, nd)),
        "reference_bh_vs_gpu_direct": dist_stats(rel(ref_bh, gpu_direct)),
        "gpu_bh_fp64_vs_gpu_direct": dist_stats(rel(gpu_bh, gpu_direct)),
        "gpu_bh_fp64_vs_reference_bh": dist_stats(rel(gpu_bh, ref_bh)),
        "gpu_direct_vs_reference_direct": dist_stats(rel(gpu_direct, ref_direct, nd)),
        "reference_seconds": {"bh_with_build": t1 - t0, "build": t_build, "direct": t2 - t1},
        "what": ("superfluid velocity vs (local term + flow + Biot-Savart + 26 images) at seeded sample "
                 "nodes; errors are |a - b| / |vs with the direct sum|; the reference's update_velocity "
                 "from oracle/_ref with its own octree (all nodes) and its direct sum (first direct_nodes)"),
    }


# ---------------------------------------------------------------- GPU side
def bench_theta(args, ov, tangle, theta: float):
    """The same 1M-point tangle at another opening angle: one RK4 step in
    each form after one untimed step, and the mixed form's error against the
    FP64 form over all nodes."""
    n = int(tangle.active.sum())
    p = params(theta)
    out = {"theta": theta, "points": n}
    vels = {}
    for name, prec in (("mixed", ov.OV_PREC_MIXED), ("fp64", ov.OV_PREC_FP64)):
        ov.configure(p, prec)
        st = ov.DeviceState(tangle.copy())
        st.run(0.0, args.dt, 1)
        st.reset_stats()
        st.run(args.dt, args.dt, 1)
        rs = st.stats()
        st.close()
        s = ov.DeviceState(tangle.copy())
        s.update_tangle(0.0)
        s.download()
        vels[name] = s.t.vels.copy()
        s.close()
        out[name] = {"ms_per_step": rs.last_run_ms, "value": n * 4 / (rs.last_run_ms / 1e3),
                     "walk_ms": rs.bs_kernel_ms / max(1.0, rs.bs_launches),
                     "cell_interactions_per_point": rs.cell_interactions / max(1.0, rs.bs_launches) / n}
    act = tangle.active
    out["mixed_over_fp64_speedup"] = out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    out["max_rel_err_mixed_vs_fp64"] = float(np.max(
        np.linalg.norm(vels["mixed"][act] - vels["fp64"][act], axis=1) /
        np.linalg.norm(vels["fp64"][act], axis=1)))
    ov.configure(params(args.theta), ov.OV_PREC_MIXED)
    return out


def bench_direct(args, ov, peak32: float, peak64: float):
    """Direct all-pairs kernel on the 22.4k-point periodic tangle: 512 rings
    in a periodic cube D = 0.1 cm, radii U[0.02, 0.05] D, dl = D/200, 26
    images.  Kernel time per evaluation (CUDA events around the kernel)
    against 43 flops per segment-point interaction, mixed and FP64."""
    from openvort_b200 import geometry as G
    from openvort_b200.tangle import Flow, Params
    D2 = 0.1
    dl2 = D2 / 200
    t = G.random_ring_tangle(args.seed + 2, 512, D2, dl=dl2, boundary="periodic-26")
    p = Params(core_a=1e-8, alpha=0.098, alpha_p=0.016, use_mf=1, dl_max=2 * dl2, hyperfriction=1,
               use_bh=0, vn=Flow("simple", {"external_v": (0.5, 0.0, 0.0)}), vs=Flow("no flow"))
    out = {"workload": f"512 rings, {int(t.active.sum())} points, periodic cube D=0.1 cm, 26 images, "
                       f"direct sum", "points": int(t.active.sum())}
    vel = {}
    for name, prec, peak in (("mixed", ov.OV_PREC_MIXED, peak32), ("fp64", ov.OV_PREC_FP64, peak64)):
        ov.configure(p, prec)
        st = ov.DeviceState(t.copy())
        st.update_tangle(0.0)
        st.reset_stats()
        for _ in range(5):
            st.update_tangle(0.0)
        rs = st.stats()
        ms = rs.bs_kernel_ms / rs.bs_launches
        inter = rs.interactions / rs.bs_launches
        tf = inter * FLOPS_P2P / (ms / 1e3) / 1e12
        out[name] = {"kernel_ms": ms, "interactions": inter, "tflops": tf, "peak_tflops": peak,
                     "frac": tf / peak if peak else None,
                     "point_evals_per_s": out["points"] / (ms / 1e3)}
        st.download()
        vel[name] = st.t.vels.copy()
        st.close()
    act = t.active
    num = np.linalg.norm(vel["mixed"][act] - vel["fp64"][act], axis=1)
    den = np.linalg.norm(vel["fp64"][act], axis=1)
    out["max_rel_err_mixed_vs_fp64"] = float(np.max(num / den))
    out["mixed_over_fp64_speedup"] = out["fp64"]["kernel_ms"] / out["mixed"]["kernel_ms"]
    return out


def bench_cfg2(args, ov):
    """The 22.4k-point periodic tangle (512 rings in a periodic cube D = 0.1
    cm, radii U[0.02, 0.05] D, dl = D/200, 26 images, counterflow 0.5 cm/s,
    alpha 0.098, alpha' 0.016) stepped with RK4 at dt = 1e-6 s, device
    resident: the direct sum and Barnes-Hut at theta = 0.4, each in FP64 and
    mixed.  The Barnes-Hut forms run the config's 500 steps; the direct sums
    a stated subset (their per-step time is steady).  Errors: Barnes-Hut vs
    direct (the approximation the reference makes) and mixed vs FP64, over
    all nodes after update_tangle."""
    from openvort_b200 import geometry as G
    from openvort_b200.tangle import Flow, Params
    D2 = 0.1
    dl2 = D2 / 200
    t = G.random_ring_tangle(args.seed + 2, 512, D2, dl=dl2, boundary="periodic-26")
    n = int(t.active.sum())
    base = Params(core_a=1e-8, alpha=0.098, alpha_p=0.016, use_mf=1, dl_max=2 * dl2, hyperfriction=1,
                  use_bh=0, bh_theta=0.4, bh_grain=1e-8, vn=Flow("simple", {"external_v": (0.5, 0.0, 0.0)}),
                  vs=Flow("no flow"))
    import dataclasses
    steps = {("direct", "fp64"): args.cfg2_direct_steps, ("direct", "mixed"): args.cfg2_direct_steps,
             ("bh", "fp64"): args.cfg2_steps, ("bh", "mixed"): args.cfg2_steps}
    out = {"workload": f"512 rings, {n} points, periodic cube D=0.1 cm, dl=D/200, 26 images, counterflow "
                       f"0.5 cm/s, RK4 dt=1e-6 s; direct sum and Barnes-Hut theta=0.4, FP64 and mixed",
           "points": n}
    vels = {}
    for method, use_bh in (("direct", 0), ("bh", 1)):
        p = dataclasses.replace(base, use_bh=use_bh)
        for form, prec in (("fp64", ov.OV_PREC_FP64), ("mixed", ov.OV_PREC_MIXED)):
            ov.configure(p, prec)
            s = ov.DeviceState(t.copy())
            s.update_tangle(0.0)
            s.download()
            vels[(method, form)] = s.t.vels.copy()
            s.close()
            k = steps[(method, form)]
            st = ov.DeviceState(t.copy())
            st.run(0.0, 1e-6, 1)
            st.reset_stats()
            st.run(1e-6, 1e-6, k)
            rs = st.stats()
            st.close()
            ms = rs.last_run_ms / k
            out[f"{method}_{form}"] = {"steps": k, "ms_per_step": ms, "rk4_steps_per_s": 1e3 / ms,
                                       "point_evals_per_s": n * 4 / (ms / 1e3)}
    act = t.active

    def rel(a, b):
        return float(np.max(np.linalg.norm(a[act] - b[act], axis=1) / np.linalg.norm(b[act], axis=1)))
    out["max_rel_err_bh_vs_direct_fp64"] = rel(vels[("bh", "fp64")], vels[("direct", "fp64")])
    out["max_rel_err_mixed_vs_fp64_direct"] = rel(vels[("direct", "mixed")], vels[("direct", "fp64")])
    out["max_rel_err_mixed_vs_fp64_bh"] = rel(vels[("bh", "mixed")], vels[("bh", "fp64")])
    out["bh_over_direct_speedup_fp64"] = out["direct_fp64"]["ms_per_step"] / out["bh_fp64"]["ms_per_step"]
    out["mixed_over_fp64_speedup_bh"] = out["bh_fp64"]["ms_per_step"] / out["bh_mixed"]["ms_per_step"]
    ov.configure(params(args.theta), ov.OV_PREC_MIXED)
    return out


def bench_cfg1(args, ov):
    """The 256-point ring (R = 1e-2 cm, open boundaries, T = 0: no mutual
    friction, a = 1.3e-8 cm, direct FP64 sum) stepped 1000 times with RK4 at
    dt = 5e-6 s, device resident, and its speed against the thin-core
    formula kappa/(4 pi R)(ln(8R/a) - 1/2).  dl_max = 2 dl keeps the
    hyperfriction threshold above the ring's curvature; with remeshing at
    [0.5, 2] dl and reconnection nothing would change on a single ring."""
    from openvort_b200 import geometry as G
    from openvort_b200.tangle import Params
    R, a, kappa, n, dt, steps = 1e-2, 1.3e-8, 9.97e-4, 256, 5e-6, args.cfg1_steps
    dl = 2 * np.pi * R / n
    p = Params(kappa=kappa, core_a=a, use_mf=0, alpha=0.0, alpha_p=0.0, hyperfriction=1, dl_max=2 * dl,
               use_bh=0)
    t = G.single_ring(n, R)
    ov.configure(p, ov.OV_PREC_FP64)
    st = ov.DeviceState(t.copy())
    st.reset_stats()
    st.run(0.0, dt, steps)
    rs = st.stats()
    st.download()
    z1 = float(st.t.pos[:, 2].mean())
    radius = float(np.mean(np.linalg.norm(st.t.pos[:, :2], axis=1)))
    st.close()
    v = z1 / (steps * dt)
    v_thin = kappa / (4 * np.pi * R) * (np.log(8 * R / a) - 0.5)
    ms = rs.last_run_ms / steps
    ov.configure(params(args.theta), ov.OV_PREC_MIXED)
    return {"workload": f"one ring, R=1e-2 cm, {n} points, open, T=0, a=1.3e-8 cm, direct FP64, RK4 "
                        f"dt=5e-6 s, {steps} steps", "steps": steps, "ms_per_step": ms,
            "rk4_steps_per_s": 1e3 / ms, "point_evals_per_s": n * 4 / (ms / 1e3),
            "ring_speed_cm_s": v, "thin_core_speed_cm_s": v_thin, "speed_over_thin_core": v / v_thin,
            "radius_drift": radius / R - 1}


def bench_batch(args, ov, peak32: float):
    """Batched ensemble: 4096 independent open-boundary ring pairs (leapfrog
    or head-on), radii U[5e-3, 2e-2] cm, U[64, 2048] points per system, mixed
    form, one persistent Biot-Savart kernel per RK4 stage, CUDA graph per
    step, autotuned kernel shape."""
    from openvort_b200 import geometry as G
    from openvort_b200.tangle import Flow, Params
    t, off, _ = G.ring_pair_ensemble(args.seed + 4, args.batch_systems, n_range=(64, 2048))
    p = Params(core_a=1e-8, alpha=0.098, alpha_p=0.016, use_mf=1, dl_max=1e-2, hyperfriction=0,
               use_bh=0, vn=Flow("no flow"), vs=Flow("no flow"))
    # the finest systems (2048 points on r = 5e-3 cm rings, spacing 3e-5 cm)
    # carry Kelvin waves of frequency ~5e6 /s at the grid scale: RK4 needs
    # dt below ~5e-7 s there
    dt = 2.5e-7
    n = int(t.active.sum())
    out = {"workload": f"{args.batch_systems} ring-pair systems, {n} points, open boundaries, direct sums per system, "
                       f"RK4 dt={dt}", "points": n, "systems": args.batch_systems, "steps": args.batch_steps}
    ov.configure(p, ov.OV_PREC_MIXED)
    b = ov.DeviceBatch(t.copy(), off)
    tu = b.autotune()
    out["tuning"] = {"targets_per_block": tu.targets_per_block, "sources_per_tile": tu.sources_per_tile,
                     "blocks_per_sm": tu.blocks_per_sm}
    b.run(0.0, dt, 2)
    b.run(2 * dt, dt, args.batch_steps)
    st = b.stats()
    ms_step = st.last_run_ms / args.batch_steps
    inter = st.interactions / st.evals
    tf = inter * FLOPS_P2P / (st.bs_kernel_ms / 1e3) / 1e12
    out.update({"value": n * 4 / (ms_step / 1e3), "unit": UNIT, "ms_per_step": ms_step,
                "rk4_steps_per_s": 1e3 / ms_step, "kernels_per_step": st.kernels_per_step,
                "bs_kernel_ms": st.bs_kernel_ms, "interactions_per_eval": inter,
                "roofline": {"bound": "fp32", "achieved": tf, "peak": peak32, "unit": "TFLOP/s",
                             "frac": tf / peak32 if peak32 else None}})
    b.close()
    # FP64 form of the same ensemble: kernel time and the mixed error
    vel = {}
    for name, prec in (("fp64", ov.OV_PREC_FP64), ("mixed", ov.OV_PREC_MIXED)):
        ov.configure(p, prec)
        bb = ov.DeviceBatch(t.copy(), off)
        bb.autotune()
        bb.update(0.0)
        bb.download()
        vel[name] = bb.t.vels.copy()
        if name == "fp64":
            out["fp64_bs_kernel_ms"] = bb.stats().bs_kernel_ms
        bb.close()
    num = np.linalg.norm(vel["mixed"] - vel["fp64"], axis=1)
    den = np.linalg.norm(vel["fp64"], axis=1)
    out["max_rel_err_mixed_vs_fp64"] = float(np.max(num / den))
    return out


def bench_adjoint(args, ov):
    """Adjoint of a 4096-point ring with Kelvin waves (modes 2-32, sigma
    1e-4 cm), alpha = 0.098, alpha' = 0.016, v_ns = 0.2 cm/s: loss =
    |centroid - target|^2 + line length after nsteps RK4 steps, checkpoints
    every 32 steps.  Gradient with respect to the initial positions and v_ns,
    FP64, against FP64 central differences along one seeded direction; the
    same gradient with the mixed forward."""
    import time as _t
    import torch
    from openvort_b200 import geometry as G
    from openvort_b200.adjoint import Adjoint, centroid_length_loss, trajectory
    from openvort_b200.tangle import Flow, Params
    n, R0 = 4096, 1e-2
    dl = 2 * np.pi * R0 / n
    # grid-scale Kelvin waves: omega ~ 2e7 /s at this spacing, so RK4 needs
    # dt ~ 5e-8 s (omega dt ~ 1)
    dt, steps, every = 5e-8, args.adjoint_steps, 32
    p = Params(kappa=9.97e-4, core_a=1e-8, use_mf=1, alpha=0.098, alpha_p=0.016, hyperfriction=1,
               max_curv_scale=0.2, hyperalpha=0.5, dl_max=dl / 2, use_bh=0,
               vn=Flow("simple", {"external_v": (0.2, 0.0, 0.0)}), vs=Flow("no flow"))
    t = G.rings_to_tangle([G.kelvin_ring(args.seed + 5, n=n, radius=R0, modes=(2, 32), sigma=1e-4)],
                          (-0.05,) * 3, (0.05,) * 3, "open")
    vn0 = np.array([0.2, 0.0, 0.0])
    target = np.array([0.0, 0.0, 0.01])
    fwd = t.links[:, 0]

    def grads(prec):
        ov.configure(p, prec)
        a = Adjoint(t)
        x0 = torch.tensor(t.pos, dtype=torch.float64, requires_grad=True)
        vn = torch.tensor(vn0, dtype=torch.float64, requires_grad=True)
        t0 = _t.perf_counter()
        xf = trajectory(a, x0, vn, 0.0, dt, steps, every)
        t1 = _t.perf_counter()
        loss = centroid_length_loss(xf, fwd, t.active, target)
        loss.backward()
        t2 = _t.perf_counter()
        return a, x0.grad.numpy().copy(), vn.grad.numpy().copy(), t1 - t0, t2 - t1

    a, gx, gv, tf, tb = grads(ov.OV_PREC_FP64)
    rng = np.random.default_rng(args.seed + 6)
    d = rng.normal(size=(n, 3)) * dl
    eps = 1e-5

    def lval_of(adj, x0, vn):
        xf = adj.forward(x0, vn, 0.0, dt, steps, every)
        return float(centroid_length_loss(torch.from_numpy(xf), fwd, t.active, target))

    def lval(x0, vn):
        return lval_of(a, x0, vn)
    fd = (lval(t.pos + eps * d, vn0) - lval(t.pos - eps * d, vn0)) / (2 * eps)
    e = np.array([1e-3, 0.0, 0.0])
    fdv = (lval(t.pos, vn0 + e) - lval(t.pos, vn0 - e)) / 2e-3
    a.close()
    # Velocity-level check at this resolution.  The reference's colinearity
    # cut-off (zero contribution when |cos - 1| < 1e-8) makes the velocity
    # discontinuous where a segment's extension passes near a target: such
    # nodes give finite differences that change with the step.  With the
    # cotangent kept off them (and their stencil neighbours) the vector-
    # Jacobian product is compared with the finite differences.
    ov.configure(p, ov.OV_PREC_FP64)
    av = Adjoint(t)
    jv = {e_: (av.velocity(t.pos + e_ * d, vn0) - av.velocity(t.pos - e_ * d, vn0)) / (2 * e_)
          for e_ in (1e-5, 1e-6)}
    scale = np.linalg.norm(jv[1e-5], axis=1)
    bad = np.linalg.norm(jv[1e-6] - jv[1e-5], axis=1) > 1e-6 * scale
    mask = bad.copy()
    for sh in (-2, -1, 1, 2):
        mask |= np.roll(bad, sh)
    gm = rng.normal(size=(n, 3))
    gm[mask] = 0
    xbm, _ = av.velocity_vjp(t.pos, gm, vn0)
    fdm = float(np.sum(gm * jv[1e-5]))
    vel_masked = abs(float(np.sum(xbm * d)) - fdm) / abs(fdm)
    av.close()
    # Trajectory-level check at the same resolution and step count with
    # smaller waves (sigma = 1e-7 cm): their slopes (~3e-4) stay below the
    # ring's own chord angle at the nearest segments, so no pair reaches the
    # cut-off and the finite differences are well defined
    ts = G.rings_to_tangle([G.kelvin_ring(args.seed + 5, n=n, radius=R0, modes=(2, 32), sigma=1e-7)],
                           (-0.05,) * 3, (0.05,) * 3, "open")
    a2 = Adjoint(ts)
    x0t = torch.tensor(ts.pos, dtype=torch.float64, requires_grad=True)
    vnt = torch.tensor(vn0, dtype=torch.float64, requires_grad=True)
    xf2 = trajectory(a2, x0t, vnt, 0.0, dt, steps, every)
    centroid_length_loss(xf2, fwd, ts.active, target).backward()

    def lval2(x0, vn):
        xf = a2.forward(x0, vn, 0.0, dt, steps, every)
        return float(centroid_length_loss(torch.from_numpy(xf), fwd, ts.active, target))
    fd2 = (lval2(ts.pos + eps * d, vn0) - lval2(ts.pos - eps * d, vn0)) / (2 * eps)
    fd2v = (lval2(ts.pos, vn0 + e) - lval2(ts.pos, vn0 - e)) / 2e-3
    smooth_pos = abs(float(np.sum(x0t.grad.numpy() * d)) - fd2) / abs(fd2)
    smooth_vns = abs(float(vnt.grad.numpy()[0]) - fd2v) / abs(fd2v)
    a2.close()
    # Trajectory-level check of config 5 as specified (sigma = 1e-4 cm) with
    # the colinearity cut-off switched off in the FP64 sums and the adjoint
    # (ov_set_colinear_cutoff(0)): the dynamics are then smooth, and the
    # adjoint and the finite differences differentiate the same function
    lib = ov.load()
    lib.ov_set_colinear_cutoff(0.0)
    try:
        a3, gx3, gv3, _, _ = grads(ov.OV_PREC_FP64)
        fd3 = (lval_of(a3, t.pos + eps * d, vn0) - lval_of(a3, t.pos - eps * d, vn0)) / (2 * eps)
        fd3v = (lval_of(a3, t.pos, vn0 + e) - lval_of(a3, t.pos, vn0 - e)) / 2e-3
        a3.close()
    finally:
        lib.ov_set_colinear_cutoff(1e-8)
    nocut_pos = abs(float(np.sum(gx3 * d)) - fd3) / abs(fd3)
    nocut_vns = abs(gv3[0] - fd3v) / abs(fd3v)
    am, gxm, gvm, tfm, tbm = grads(ov.OV_PREC_MIXED)
    am.close()
    ov.configure(p, ov.OV_PREC_FP64)
    ad = float(np.sum(gx * d))
    return {"workload": f"ring R=1e-2 cm, {n} points, Kelvin modes 2-32 (sigma 1e-4 cm), {steps} RK4 steps "
                        f"dt={dt}, checkpoints every {every}", "points": n, "steps": steps,
            "forward_s": tf, "backward_s": tb, "mixed_forward_s": tfm, "mixed_backward_s": tbm,
            "fd_rel_err_positions": abs(ad - fd) / abs(fd), "fd_rel_err_vns": abs(gv[0] - fdv) / abs(fdv),
            "mixed_fd_rel_err_positions": abs(float(np.sum(gxm * d)) - fd) / abs(fd),
            "mixed_fd_rel_err_vns": abs(gvm[0] - fdv) / abs(fdv),
            "velocity_vjp_fd_rel_err_masked": vel_masked, "discontinuous_nodes": int(bad.sum()),
            "fd_rel_err_positions_small_waves": smooth_pos, "fd_rel_err_vns_small_waves": smooth_vns,
            "fd_rel_err_positions_no_colinear_cutoff": nocut_pos, "fd_rel_err_vns_no_colinear_cutoff": nocut_vns,
            "note": "fd_rel_err_* at 4096 points include the jumps of the reference's colinearity "
                    "cut-off crossed between the perturbed runs; *_no_colinear_cutoff: the same input, "
                    "FP64, with that cut-off switched off in the sums and the adjoint"}


def bench_reconnect(args, ov, tangle, p):
    """One vortex-vortex reconnection pass on the 1M-point tangle at the
    0.087 rad angle cut-off: the GPU pair search and the whole pass (host
    loop over the candidates with the approach test on the GPU).  rec_dist
    is the tangle's point spacing DL (5e-4 cm): the reference's defaults pair
    rec_dist = dl_min = 1e-3 cm with a remesh that keeps the spacing above
    dl_min, so only nodes of different lines (or far along one line) are
    candidates; a rec_dist of twice the spacing would also make every second
    neighbour on the small rings a candidate.  The reference's O(N^2) pair
    loop is timed on a 20k-point tangle of the same generator and scaled by
    N^2."""
    import time as _t
    lib = ov.load()
    rec_dist, rec_angle = DL, 0.087
    ov.configure(p, ov.OV_PREC_FP64)
    ht = tangle.copy()
    ov.update_tangle(ht, 0.0)       # tangents of the current positions
    lib.ov_reconnect_candidates(ht.ptr(), rec_dist, rec_angle, None, 0)   # warm-up
    t0 = _t.perf_counter()
    ncand = lib.ov_reconnect_candidates(ht.ptr(), rec_dist, rec_angle, None, 0)
    t_search = _t.perf_counter() - t0
    hc = ht.copy()
    hc.set_images_from_library(lib)
    hc.recalc[:] = 0
    t0 = _t.perf_counter()
    nrec = lib.ov_reconnect_vortices(hc.ptr(), 0.0, rec_dist, rec_angle)
    t_pass = _t.perf_counter() - t0
    from openvort_b200._lib import ReconnectStats
    st = ReconnectStats()
    lib.ov_reconnect_get_stats(C.byref(st))
    out = {"workload": f"{int(tangle.active.sum())} points, rec_dist={rec_dist}, rec_angle={rec_angle}",
           "candidates": ncand, "reconnections": nrec, "gpu_search_s": t_search, "gpu_pass_s": t_pass,
           "tested": st.tested, "nodes_summed": st.nodes_summed, "sums_s": st.sums_s,
           "upload_and_search_s": st.search_s}
    # mixed form: FP32 far-field sums with an error bound per node, FP64
    # again where the bound leaves the approach test's sign open
    ov.configure(p, ov.OV_PREC_MIXED)
    hm = ht.copy()
    hm.set_images_from_library(lib)
    hm.recalc[:] = 0
    t0 = _t.perf_counter()
    nrec_m = lib.ov_reconnect_vortices(hm.ptr(), 0.0, rec_dist, rec_angle)
    t_mixed = _t.perf_counter() - t0
    ov.configure(p, ov.OV_PREC_FP64)
    st = ReconnectStats()
    lib.ov_reconnect_get_stats(C.byref(st))
    act = hc.active
    dv = np.linalg.norm(hm.vels[act] - hc.vels[act], axis=1) / np.maximum(np.linalg.norm(hc.vels[act], axis=1),
                                                                           1e-300)
    out["mixed"] = {"gpu_pass_s": t_mixed, "reconnections": nrec_m, "tested": st.tested,
                    "nodes_summed": st.nodes_summed, "fp64_rechecks": st.fp64_rechecks, "sums_s": st.sums_s,
                    "upload_and_search_s": st.search_s,
                    "same_links_as_fp64": bool(np.array_equal(hm.links, hc.links) and nrec_m == nrec),
                    "max_rel_err_vels_vs_fp64": float(dv.max()) if dv.size else 0.0,
                    "speedup_over_fp64_pass": t_pass / t_mixed if t_mixed > 0 else None}
    from oracle.oracle import Ref, have_ref
    if have_ref():
        small, _ = make_tangle(20000, args.seed + 7)
        ref = Ref(threads=os.cpu_count())
        rs = ref.update_tangle(small, p, 0.0)
        t0 = _t.perf_counter()
        ref.reconnect(rs, p, 0.0, rec_dist, rec_angle)
        t_ref = _t.perf_counter() - t0
        ns, nb = int(small.active.sum()), int(tangle.active.sum())
        out["reference_pass_s_20k"] = t_ref
        out["reference_pass_s_estimate"] = t_ref * (nb / ns) ** 2
        out["reference_note"] = "reference reconnect() on a 20k-point tangle (one thread: its loop is serial), scaled by N^2"
    return out


def bench_remesh(args, ov):
    """One remesh pass (ov_remesh, host tangle in and out) on a 1M-point
    tangle with uneven resolution: 0.2% of the nodes pushed 30-80% of the
    way to their forward neighbour, 500 pairs of nodes taken out;
    min_dist = 0.6 dl, max_dist = 2.5 dl (the reference's defaults have a
    1:5 ratio).  The reference's remesh, which recomputes every tangent after
    each change, is timed on a 20k-point tangle of the same generator and
    perturbation density and scaled by N^2."""
    import time as _t
    from openvort_b200 import geometry as G
    lib = ov.load()
    p = params(args.theta)
    ov.configure(p, ov.OV_PREC_FP64)
    lo, hi = 0.6 * DL, 2.5 * DL
    t, _ = make_tangle(args.points, args.seed + 11, empty_slots=20000)
    n = int(t.active.sum())
    G.perturb_spacing(t, args.seed + 11, frac_move=0.002, n_gaps=n // 2000)
    ov.update_tangents_normals(t)
    warm = t.copy()
    lib.ov_remesh(warm.ptr(), lo, hi, None)
    run = t.copy()
    t0 = _t.perf_counter()
    changes = lib.ov_remesh(run.ptr(), lo, hi, None)
    t_pass = _t.perf_counter() - t0
    if changes < 0:
        raise SystemExit(f"ov_remesh: {lib.ov_last_error_message().decode()}")
    out = {"workload": f"{n} points, 0.2% of the nodes moved along the line, {n // 2000} node pairs "
                       f"taken out, min_dist={lo:g}, max_dist={hi:g}",
           "changes": changes, "gpu_pass_s": t_pass,
           "path": "ov_remesh on a struct tangle_state in host memory (upload, GPU scan, host loop over "
                   "the changes, GPU tangents near them, GPU enforce_boundaries, changed nodes back)"}
    from oracle.oracle import Ref, have_ref
    if have_ref():
        small, _ = make_tangle(20000, args.seed + 11, empty_slots=400)
        ns = int(small.active.sum())
        G.perturb_spacing(small, args.seed + 11, frac_move=0.002, n_gaps=ns // 2000)
        ref = Ref(threads=1)
        rs = ref.update_tangents_normals(small, p)
        t0 = _t.perf_counter()
        ref.remesh(rs, p, lo, hi)
        t_ref = _t.perf_counter() - t0
        out["reference_pass_s_20k"] = t_ref
        out["reference_pass_s_estimate"] = t_ref * (n / ns) ** 2
        out["reference_note"] = ("reference remesh() on a 20k-point tangle (serial: each change runs "
                                 "update_tangents_normals over all nodes), scaled by N^2")
    return out


def bench_frames(args, ov, tangle, p):
    """Frames of the 1M-point state: the time until ov_state_save_frame
    returns (device snapshot queued) and until the file is on disk, text
    (the reference's format) and binary (with the time stamp); the
    reference's save_tangle timed on a 200k-point tangle and scaled by N
    (its loop is linear and serial)."""
    import shutil
    import time as _t
    lib = ov.load()
    ov.configure(p, ov.OV_PREC_FP64)
    t = tangle.copy()
    st = ov.DeviceState(t)
    st.update_tangle(0.0)
    n = int(t.active.sum())
    out = {"workload": f"{n} points, frames of a device-resident state"}
    tmp = tempfile.mkdtemp(prefix="ovframes")
    try:
        for name, binary in (("binary", True), ("text", False)):
            path = os.path.join(tmp, f"frame.{name}")
            st.save_frame(path, 0.0, binary=binary)      # warm-up (buffers)
            st.wait_frames()
            t0 = _t.perf_counter()
            st.save_frame(path, 0.0, binary=binary)
            t1 = _t.perf_counter()
            st.wait_frames()
            t2 = _t.perf_counter()
            out[name] = {"call_s": t1 - t0, "written_s": t2 - t0, "bytes": os.path.getsize(path)}
        from oracle.oracle import Ref, have_ref
        if have_ref():
            small, _ = make_tangle(200000, args.seed + 3)
            st2 = ov.DeviceState(small)
            st2.update_tangle(0.0)
            st2.download()
            st2.close()
            ref = Ref()
            f = ref.lib.save_tangle
            f.restype = None
            f.argtypes = [C.c_char_p, C.c_void_p]
            t0 = _t.perf_counter()
            f(os.path.join(tmp, "ref.dat").encode(), C.cast(small.ptr(), C.c_void_p))
            t_ref = _t.perf_counter() - t0
            ns = int(small.active.sum())
            out["reference_text_s_200k"] = t_ref
            out["reference_text_s_estimate"] = t_ref * n / ns
    finally:
        st.close()
        shutil.rmtree(tmp, ignore_errors=True)
    out["host_threads"] = os.cpu_count()
    return out


def independent_tangles(args, ov, p, dist, rank, world):
    """Weak-scaling figures beside the sharded headline: every rank steps its
    own seeded tangle of the same size, no collective on the data path."""
    from openvort_b200.dist import rank_seed
    t, _ = make_tangle(args.points, rank_seed(args.seed, rank))
    n = int(t.active.sum())
    ov.configure(p, ov.OV_PREC_MIXED)
    st = ov.DeviceState(t.copy())
    st.run(0.0, args.dt, 1)
    barrier(dist)
    st.reset_stats()
    barrier(dist)
    st.run(args.dt, args.dt, args.steps)
    barrier(dist)
    ms = max_over_ranks(dist, st.stats().last_run_ms) / args.steps
    st.close()
    from openvort_b200.dist import sum_over_ranks
    n_job = int(round(sum_over_ranks(dist, float(n))))
    return {"scaling": "weak", "points_all_ranks": n_job, "ms_per_step": ms,
            "value": n_job * 4 / (ms / 1e3), "unit": UNIT,
            "parallelism": f"{world} independent tangles (one per GPU), no collective on the data path"}


def run_sharded(args, world, rank, local, dist):
    """One tangle over all ranks (openvort_b200.shard): every rank holds the
    same tangle and builds the same tree, walks its share of the targets, and
    the Biot-Savart sums (48 bytes per node) are all-gathered in place at each
    evaluation.  Strong scaling: the whole job is one tangle."""
    import torch
    import openvort_b200 as ov
    from openvort_b200 import dist as D
    from openvort_b200.shard import ShardedRun

    lib = ov.load()
    if lib.ov_init(local) != 0:
        raise SystemExit(f"libov_gpu: {lib.ov_last_error_message().decode()}")
    torch.cuda.set_device(local)
    p = params(args.theta)
    tangle, n_rings = make_tangle(args.points, args.seed)
    n = int(tangle.active.sum())
    ov.configure(p, ov.OV_PREC_MIXED)
    st = ov.DeviceState(tangle.copy())
    run = ShardedRun(st, dist)
    run.run(0.0, args.dt, args.warmup)
    barrier(dist)
    st.reset_stats()
    clocks = Clocks(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(dist)
    e0.record()
    # every stage synchronises the library's stream and the exchange's, so
    # the events bracket the whole run
    run.run(args.warmup * args.dt, args.dt, args.steps)
    e1.record()
    e1.synchronize()
    barrier(dist)
    clk = clocks.stop()
    ms_run = max_over_ranks(dist, e0.elapsed_time(e1))
    rs = st.stats()
    walk_ms = max_over_ranks(dist, rs.bs_kernel_ms / max(1.0, rs.bs_launches))
    cells = D.sum_over_ranks(dist, rs.cell_interactions)
    p2p = D.sum_over_ranks(dist, rs.interactions)
    launches = int(rs.launches)
    # end to end through the public API: each step uploads the tangle from
    # pinned host memory, runs the sharded step and reads the positions back
    e2e = None
    if not args.no_e2e:
        alloc, keep = pinned_alloc()
        ht = tangle.copy(alloc=alloc)
        st.t = ht
        barrier(dist)
        t0 = time.perf_counter()
        tt = (args.warmup + args.steps) * args.dt
        for _ in range(args.steps):
            st.upload()
            run.step(tt, args.dt)
            st.download(ov.OV_FIELD_POS)
            tt += args.dt
        barrier(dist)
        sec = max_over_ranks(dist, time.perf_counter() - t0)
        e2e = {"value": n * 4 * args.steps / sec, "unit": UNIT, "h2d_bytes_per_step": ht.n * (24 + 8 + 8),
               "d2h_bytes_per_step": ht.n * 24, "ms_per_step": sec / args.steps * 1e3,
               "path": "DeviceState.upload from pinned host memory + sharded RK4 step + positions read back"}
    st.close()
    indep = None if args.no_extra or world == 1 else independent_tangles(args, ov, p, dist, rank, world)
    if rank == 0:
        ms_step = ms_run / args.steps
        peak32 = C.c_double(0)
        lib.ov_measure_fma_peak(0, C.byref(peak32))
        launches_walk = max(1.0, rs.bs_launches)
        flops = (p2p * FLOPS_P2P + cells * FLOPS_CELL) / launches_walk
        achieved = flops / (walk_ms / 1e3) / 1e12 / world
        print(json.dumps({
            "metric": METRIC, "value": n * 4 * args.steps / (ms_run / 1e3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": f"large periodic tangle: {n} points ({n_rings} rings, D=0.4 cm, dl=D/800, "
                                   f"radii U[0.02,0.05]D), 26 periodic images, Barnes-Hut theta={args.theta}, "
                                   f"mixed FP32/FP64, RK4 dt={args.dt}",
                       "points": n, "points_all_ranks": n, "theta": args.theta, "images": 26, "dt": args.dt,
                       "parallelism": f"one tangle over {world} ranks: each walks 1/{world} of the targets "
                                      f"in tree key order, Biot-Savart sums all-gathered per evaluation",
                       "l2": "working set (octree cells + node table) larger than the 126 MB L2"},
            "rk4_steps_per_s": 1e3 / ms_step,
            "walk_ms_per_launch_max_over_ranks": walk_ms,
            "cell_interactions_per_point": cells / launches_walk / n,
            "exchange_bytes_per_evaluation": 48 * n,
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak32.value, "unit": "TFLOP/s",
                         "frac": achieved / peak32.value if peak32.value else None, "traffic": None,
                         "kernel": "Barnes-Hut walk, one rank's share of the targets (slowest rank)",
                         "peak_source": "ov_measure_fma_peak: FP32 FMA burst on this GPU, this run"},
            "independent_tangles": indep,
            "process_group": D.describe(dist),
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
        }))
    D.close(dist)


def main():
    args = parse()
    world, rank, local, dist = dist_setup(args)
    if args.impl == "reference":
        if rank == 0:
            run_reference_arm(args, world, rank)
        from openvort_b200 import dist as D
        D.close(dist)
        return
    if args.shard or (world > 1 and not args.independent):
        run_sharded(args, world, rank, local, dist)
        return

    import torch
    import openvort_b200 as ov
    from openvort_b200 import _lib

    lib = ov.load()
    if lib.ov_init(local) != 0:
        raise SystemExit(f"libov_gpu: {lib.ov_last_error_message().decode()}")
    torch.cuda.set_device(local)
    p = params(args.theta)
    if args.only and args.only not in ("walk", "walk64"):
        peak32, peak64 = C.c_double(0), C.c_double(0)
        lib.ov_measure_fma_peak(0, C.byref(peak32))
        lib.ov_measure_fma_peak(1, C.byref(peak64))
        part = {"direct": lambda: bench_direct(args, ov, peak32.value, peak64.value),
                "batch": lambda: bench_batch(args, ov, peak32.value),
                "cfg2": lambda: bench_cfg2(args, ov),
                "adjoint": lambda: bench_adjoint(args, ov)}
        if args.only == "reconnect":
            t, _ = make_tangle(args.points, args.seed)
            out = bench_reconnect(args, ov, t, p)
        else:
            out = part[args.only]()
        print(json.dumps({"only": args.only, args.only: out}))
        from openvort_b200 import dist as D
        D.close(dist)
        return
    from openvort_b200.dist import rank_seed
    tangle, n_rings = make_tangle(args.points, rank_seed(args.seed, rank))
    n = int(tangle.active.sum())
    # every rank its own tangle: the job's points are the sum over ranks
    from openvort_b200.dist import sum_over_ranks
    n_job = int(round(sum_over_ranks(dist, float(n))))

    # ---------------- device-resident timing, mixed precision (FP64 for
    # --only walk64, which profiles the FP64 walk alone)
    ov.configure(p, ov.OV_PREC_FP64 if args.only == "walk64" else ov.OV_PREC_MIXED)
    st = ov.DeviceState(tangle.copy())
    st.run(0.0, args.dt, args.warmup)
    barrier(dist)
    st.reset_stats()
    clocks = Clocks(local)
    clocks.start()
    barrier(dist)
    st.run(args.warmup * args.dt, args.dt, args.steps)
    barrier(dist)
    clk = clocks.stop()
    rs = st.stats()
    ms_run = max_over_ranks(dist, rs.last_run_ms)
    ms_step = ms_run / args.steps
    value = n_job * 4 * args.steps / (ms_run / 1e3)
    # roofline of the Barnes-Hut walk: algorithmic flops per launch / device
    # time per launch (CUDA events around each walk launch on its stream)
    flops = rs.interactions * FLOPS_P2P + rs.cell_interactions * FLOPS_CELL
    walk_ms = rs.bs_kernel_ms / max(1.0, rs.bs_launches)
    achieved = flops / max(1.0, rs.bs_launches) / (walk_ms / 1e3) / 1e12
    peak32 = C.c_double(0)
    lib.ov_measure_fma_peak(0, C.byref(peak32))
    launches = int(rs.launches)
    walk_share = rs.bs_kernel_ms / ms_run if ms_run > 0 else None
    build_share = rs.build_ms / ms_run if ms_run > 0 else None
    st.close()
    if args.only in ("walk", "walk64"):
        print(json.dumps({"only": args.only, "points": n, "ms_per_step": ms_step, "walk_ms": walk_ms,
                          "achieved_tflops": achieved, "peak_tflops": peak32.value,
                          "frac": achieved / peak32.value if peak32.value else None,
                          "cell_interactions_per_point": rs.cell_interactions / max(1.0, rs.bs_launches) / n}))
        from openvort_b200 import dist as D
        D.close(dist)
        return

    # ---------------- plain FP64 form, same workload
    ov.configure(p, ov.OV_PREC_FP64)
    st64 = ov.DeviceState(tangle.copy())
    st64.run(0.0, args.dt, 1)
    barrier(dist)
    st64.reset_stats()
    barrier(dist)
    st64.run(args.dt, args.dt, args.fp64_steps)
    barrier(dist)
    rs64 = st64.stats()
    ms64 = max_over_ranks(dist, rs64.last_run_ms) / args.fp64_steps
    value64 = n_job * 4 / (ms64 / 1e3)
    peak64 = C.c_double(0)
    lib.ov_measure_fma_peak(1, C.byref(peak64))
    flops64 = rs64.interactions * FLOPS_P2P + rs64.cell_interactions * FLOPS_CELL
    ach64 = flops64 / max(1.0, rs64.bs_launches) / (rs64.bs_kernel_ms / max(1.0, rs64.bs_launches) / 1e3) / 1e12
    st64.close()

    # ---------------- accuracy: mixed vs FP64 (all nodes), and both vs an
    # FP64 direct sum (no tree) on 4096 seeded sample nodes
    err = {}
    if rank == 0:
        def vel(prec):
            ov.configure(p, prec)
            s = ov.DeviceState(tangle.copy())
            s.update_tangle(0.0)
            s.download()
            v, vsf = s.t.vels.copy(), s.t.vs.copy()
            s.close()
            return v, vsf
        (v64, vs64), (vmx, _) = vel(ov.OV_PREC_FP64), vel(ov.OV_PREC_MIXED)
        act = tangle.active
        num = np.linalg.norm(vmx[act] - v64[act], axis=1)
        den = np.linalg.norm(v64[act], axis=1)
        err["max_rel_err_mixed_vs_fp64"] = float(np.max(num / den))
        rng = np.random.default_rng(4096)
        idx = rng.choice(np.nonzero(act)[0], size=min(4096, int(act.sum())), replace=False).astype(np.int32)
        pts = tangle.pos[idx]
        ov.configure(p, ov.OV_PREC_FP64)
        s = ov.DeviceState(tangle.copy())
        direct = s.eval_points(pts, idx, method=0)
        bh64 = s.eval_points(pts, idx, method=1)
        ov.configure(p, ov.OV_PREC_MIXED)
        s2 = ov.DeviceState(tangle.copy())
        bhmx = s2.eval_points(pts, idx, method=1)
        s.close()
        s2.close()
        # superfluid velocity with the FP64 direct Biot-Savart sum at the
        # sample nodes: local term + external + direct sum
        vs_direct = vs64[idx] - bh64 + direct
        ref_norm = np.linalg.norm(vs_direct, axis=1)

        def rel(a, b):
            return float(np.max(np.linalg.norm(a - b, axis=1) / ref_norm))
        err["vs_rel_err_bh_fp64_vs_direct_4096"] = rel(bh64, direct)
        err["vs_rel_err_bh_mixed_vs_direct_4096"] = rel(bhmx, direct)
        err["vs_rel_err_bh_mixed_vs_bh_fp64_4096"] = rel(bhmx, bh64)
        if world == 1 and not args.no_cpu_baseline:
            err["bh_vs_direct_reference_4096"] = bh_reference_check(tangle, p, idx, bh64, direct, vs64)

    # ---------------- end to end through the reference-named C ABI, pinned
    # host buffers: update_tangle + rk4_step copy in and out every call
    e2e = None
    if not args.no_e2e:
        alloc, keep = pinned_alloc()
        ht = tangle.copy(alloc=alloc)
        ov.configure(p, ov.OV_PREC_MIXED)
        ov.update_tangle(ht, 0.0)
        ov.rk4_step(ht, 0.0, args.dt)
        barrier(dist)
        t0 = time.perf_counter()
        tt = args.dt
        for _ in range(args.steps):
            ov.update_tangle(ht, tt)
            ov.rk4_step(ht, tt, args.dt)
            tt += args.dt
        barrier(dist)
        sec = max_over_ranks(dist, time.perf_counter() - t0)
        N = ht.n
        h2d = N * (40 + 88 + 64)      # geometry, velocities, rk4 inputs
        d2h = N * (56 + 48 + 24)      # dxi+tangents+normals, vels+vs, positions
        e2e = {"value": n_job * 4 * args.steps / sec, "unit": UNIT, "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": sec / args.steps * 1e3,
               "path": "update_tangents_normals + update_velocities + rk4_step over struct tangle_state "
                       "in pinned host memory"}

    direct = batch = adjoint = reconnection = remeshing = frames = theta_alt = cfg1 = cfg2 = None
    # the single-GPU objects (and their CPU reference samples) belong to the
    # 1-GPU line; a multi-GPU run measures the headline path only
    if not args.no_extra and world == 1:
        theta_alt = bench_theta(args, ov, tangle, 0.3 if args.theta != 0.3 else 0.5)
        direct = bench_direct(args, ov, peak32.value, peak64.value)
        cfg2 = bench_cfg2(args, ov)
        cfg1 = bench_cfg1(args, ov)
        batch = bench_batch(args, ov, peak32.value)
        adjoint = bench_adjoint(args, ov)
        reconnection = bench_reconnect(args, ov, tangle, p)
        remeshing = bench_remesh(args, ov)
        frames = bench_frames(args, ov, tangle, p)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_sample(tangle, p, target_s=10.0)

    # DRAM bytes (read + write) per walk launch, from the ncu capture of this
    # kernel on this workload, scaled by the points per launch
    traffic = WALK_DRAM_BYTES_PER_POINT * n if WALK_DRAM_BYTES_PER_POINT else None

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": bench_config(args, n, n_job, n_rings, world),
            "rk4_steps_per_s": world * 1e3 / ms_step,
            "fp64": {"value": value64, "ms_per_step": ms64, "rk4_steps_per_s": world * 1e3 / ms64,
                     "roofline_frac_of_fp64_peak": ach64 / peak64.value if peak64.value else None,
                     "fp64_fma_peak_tflops": peak64.value},
            "mixed_over_fp64_speedup": ms64 / ms_step,
            **err,
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak32.value, "unit": "TFLOP/s",
                         "frac": achieved / peak32.value if peak32.value else None, "traffic": traffic,
                         "traffic_source": WALK_TRAFFIC_SOURCE,
                         "kernel": "k_walk_multi<mixed> (Barnes-Hut walk, one traversal per point for all 27 images)",
                         "peak_source": "ov_measure_fma_peak: FP32 FMA burst on this GPU, this run",
                         "flops_per_launch": flops / max(1.0, rs.bs_launches),
                         "launch_ms": walk_ms, "share_of_step": walk_share,
                         "p2p_interactions_per_point": rs.interactions / max(1.0, rs.bs_launches) / n,
                         "cell_interactions_per_point": rs.cell_interactions / max(1.0, rs.bs_launches) / n,
                         "cell_visits_per_warp": rs.warp_iterations / max(1.0, rs.bs_launches) / (n / 32.0),
                         "hbm": ({"achieved_gbs": traffic / (walk_ms / 1e3) / 1e9, "peak_gbs": HBM_PEAK,
                                  "frac": traffic / (walk_ms / 1e3) / 1e9 / HBM_PEAK,
                                  "peak_source": HBM_PEAK_SOURCE + " copy bandwidth"}
                                 if traffic else None),
                         "tree_build_share_of_step": build_share},
            "other_theta": theta_alt,
            "direct_22k": direct,
            "cfg2_22k": cfg2,
            "cfg1_ring": cfg1,
            "batch_4096": batch,
            "adjoint_4096": adjoint,
            "reconnection_1m": reconnection,
            "remesh_1m": remeshing,
            "frames_1m": frames,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
        }
        print(json.dumps(line))
    from openvort_b200 import dist as D
    D.close(dist)


if __name__ == "__main__":
    main()
