"""The reference's main loop as a program (oracle/linked_main.c), built from
the reference's sources unmodified (oracle/_ref/ov_linked_ref) and linked
against libov_gpu.so by the integration recipe (oracle/_ref/ov_linked_gpu):
input and output files."""
from __future__ import annotations

import struct
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
REF_EXE = ROOT / "oracle" / "_ref" / "ov_linked_ref"
GPU_EXE = ROOT / "oracle" / "_ref" / "ov_linked_gpu"
WALLS = {"periodic-26": [1] * 6, "open": [0] * 6}


def write_input(path, t, steps, use_bh, theta, dt, rec_dist, rec_angle, dl_min, dl_max, core_a, alpha,
                alpha_p, vn):
    n = t.n
    with open(path, "wb") as f:
        f.write(struct.pack("<3i", n, steps, use_bh))
        f.write(struct.pack("<18d", theta, dt, rec_dist, rec_angle, dl_min, dl_max, core_a, alpha, alpha_p,
                            *vn, *t.box_lo, *t.box_hi))
        f.write(struct.pack("<6i", *WALLS[t.boundary]))
        f.write(t.boundary.encode().ljust(32, b"\0"))
        f.write(np.ascontiguousarray(t.pos, dtype="<f8").tobytes())
        for col in (t.links[:, 0], t.links[:, 1], t.stat[:, 0], t.stat[:, 1]):
            f.write(np.ascontiguousarray(col, dtype="<i4").tobytes())


def read_output(path):
    b = Path(path).read_bytes()
    n, recs = struct.unpack_from("<2i", b, 0)
    o = 8
    pos = np.frombuffer(b, "<f8", 3 * n, o).reshape(n, 3)
    o += 24 * n
    fwd, rev, st = (np.frombuffer(b, "<i4", n, o + 4 * n * i) for i in range(3))
    return {"n": n, "recs": recs, "pos": pos, "fwd": fwd, "rev": rev, "status": st}


def run(exe, inp, out):
    r = subprocess.run([str(exe), str(inp), str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (exe, r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    return read_output(out)
