"""GPU: bench.py's code paths run to the end on a small tangle and print
one JSON line with the contract's keys: the default single-GPU line and the
sharded one-tangle line (one rank here; more ranks run the same code with
NCCL between them).  The numbers are not checked."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
KEYS = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
        "scaling", "dtype", "data", "config")


def run_bench(*args, timeout=600):
    env = dict(os.environ)
    env.pop("WORLD_SIZE", None)
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout[-2000:]
    return json.loads(lines[0])


def test_default_line_small_tangle():
    d = run_bench("--points", "20000", "--steps", "3", "--warmup", "3", "--no-extra", "--no-cpu-baseline")
    for k in KEYS + ("roofline", "e2e", "gpu_launches", "clocks"):
        assert k in d, k
    assert d["n_gpus"] == 1 and d["value"] > 0 and d["e2e"]["value"] > 0
    assert d["gpu_launches"] > 0


def test_sharded_line_small_tangle():
    d = run_bench("--shard", "--points", "20000", "--steps", "2", "--warmup", "3")
    for k in KEYS + ("roofline", "e2e", "process_group", "gpu_launches"):
        assert k in d, k
    assert d["scaling"] == "strong" and d["value"] > 0 and d["e2e"]["value"] > 0
