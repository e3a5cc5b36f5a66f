"""Build libov_gpu.so (the CUDA product) in-tree for sm_100a.

    python -m openvort_b200.build          # or openvort_b200.build.build()

Each .cu under csrc/ is compiled with nvcc for sm_100a only, then linked into
openvort_b200/libov_gpu.so with the CUDA runtime linked statically, so the
library loads on any machine with the driver and needs no JIT cache.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD_DIR = PKG / "_build"
LIB = PKG / "libov_gpu.so"
SOURCES = ["ov_api.cu", "ov_geom.cu", "ov_direct.cu", "ov_tree.cu", "ov_walk.cu", "ov_peak.cu",
           "ov_noalloc.cu", "ov_batch.cu", "ov_adjoint.cu", "ov_reconnect.cu",
           "ov_remesh.cu", "ov_frames.cu", "ov_loops.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2",
                     "-I", str(ROOT / "include"), "-I", str(CSRC)]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libov_gpu.so")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, extra_flags: list[str] | None = None) -> Path:
    """Compile every kernel source and link libov_gpu.so; returns its path."""
    BUILD_DIR.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "openvort_b200.h"]
    flags = NVCC_FLAGS + (extra_flags or [])
    jobs = []
    for src in SOURCES:
        s = CSRC / src
        o = BUILD_DIR / (s.stem + ".o")
        if _stale(o, [s] + headers):
            jobs.append([nvcc(), *flags, "-c", str(s), "-o", str(o)])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed ({r.returncode}):\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout, r.stderr, flush=True)

    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(run, jobs))
    objs = [BUILD_DIR / (Path(s).stem + ".o") for s in SOURCES]
    if jobs or _stale(LIB, objs):
        run([nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-cudart", "static",
             "-Xlinker", "--no-undefined"])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
