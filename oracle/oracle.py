"""ctypes access to the CPU checkers.  TEST INFRASTRUCTURE ONLY: imported by
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg, never by the
product.

  Oracle  - liboracle.so, this repository's C restatement (ov_oracle.c)
  Ref     - _ref/libov_ref.so, the unmodified reference compiled from its own
            sources (oracle/Makefile); present wherever it was built

Both take an openvort_b200.tangle.HostTangle and Params and write their
results into a copy of the tangle, leaving the input untouched.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from openvort_b200.tangle import FLOW_KINDS, FLOW_PARAMS, IMAGE_TABLES, HostTangle, Params

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libov_ref.so"
# the reference checkout the recipe compiles from: $OPENVORT_REF, by default
# the read-only checkout of the machine that builds the checkers
REF_SRC = Path(os.environ.get("OPENVORT_REF", "/root/reference"))


def build(ref: bool = True):
    """Compile liboracle.so, and _ref/libov_ref.so with the linked main-loop
    programs when the reference sources are present; elsewhere the prebuilt
    files are used."""
    targets = ["liboracle.so"]
    if ref and (REF_SRC / "src" / "tangle.c").exists():
        # the reference library, and its main loop built unmodified and
        # linked against libov_gpu.so (which must be built first)
        targets += ["ref", "linked"]
    subprocess.run(["make", "-s", "-C", str(HERE), f"REF={REF_SRC}", *targets], check=True)


# ---------------------------------------------------------------- restatement
class OvoFlow(C.Structure):
    _fields_ = [("kind", C.c_int), ("s", C.c_double * 4), ("v", (C.c_double * 3) * 2)]


class OvoTangle(C.Structure):
    _fields_ = [("n", C.c_int), ("pos", C.c_void_p), ("fwd", C.c_void_p), ("rev", C.c_void_p),
                ("status", C.c_void_p), ("pin_wall", C.c_void_p), ("lo", C.c_double * 3),
                ("hi", C.c_double * 3), ("wall", C.c_int * 6), ("n_img", C.c_int),
                ("img", C.c_void_p)]


class OvoParams(C.Structure):
    _fields_ = [("kappa", C.c_double), ("core_a", C.c_double), ("lia_only", C.c_int),
                ("use_bh", C.c_int), ("bh_quadtree", C.c_int), ("bh_theta", C.c_double),
                ("bh_grain", C.c_double), ("use_mf", C.c_int), ("alpha", C.c_double),
                ("alpha_p", C.c_double), ("hyperfriction", C.c_int),
                ("max_curv_scale", C.c_double), ("hyperalpha", C.c_double),
                ("dl_max", C.c_double), ("rk4_classic", C.c_int), ("vn", OvoFlow),
                ("vs", OvoFlow), ("vb", OvoFlow)]


def _flow(f) -> OvoFlow:
    o = OvoFlow()
    o.kind = FLOW_KINDS.index(f.name)
    si = vi = 0
    spec = FLOW_PARAMS[f.name]
    # scalar / vector slots in each flow's parameter-list order
    for pname, ptype in spec:
        val = f.params.get(pname, 0.0)
        if ptype == 2:
            o.v[vi][:] = [float(x) for x in val]
            vi += 1
        else:
            o.s[si] = float(val)
            si += 1
    return o


class Oracle:
    def __init__(self, path: Path = ORACLE_SO):
        if not Path(path).exists():
            build(ref=False)
        self.lib = C.CDLL(str(path))
        for name in ("ovo_tangents_normals", "ovo_velocities", "ovo_segments_at", "ovo_bh_at",
                     "ovo_rk4_step", "ovo_update_tangle"):
            getattr(self.lib, name).restype = None

    @staticmethod
    def _tangle(t: HostTangle, pos=None):
        o = OvoTangle()
        keep = []
        p = np.ascontiguousarray(t.pos if pos is None else pos)
        fwd = np.ascontiguousarray(t.links[:, 0])
        rev = np.ascontiguousarray(t.links[:, 1])
        st = np.ascontiguousarray(t.stat[:, 0])
        pw = np.ascontiguousarray(t.stat[:, 1])
        table = IMAGE_TABLES[t.boundary]
        img = np.array([[*s, r] for s, r in table], dtype=np.int32).reshape(-1, 4)
        keep += [p, fwd, rev, st, pw, img]
        o.n = t.n
        o.pos, o.fwd, o.rev = p.ctypes.data, fwd.ctypes.data, rev.ctypes.data
        o.status, o.pin_wall = st.ctypes.data, pw.ctypes.data
        o.lo[:] = t.box_lo
        o.hi[:] = t.box_hi
        o.wall[:] = t.walls
        o.n_img = len(table)
        o.img = img.ctypes.data if len(table) else None
        return o, keep

    @staticmethod
    def _params(p: Params, rk4_classic=False) -> OvoParams:
        o = OvoParams()
        for name in ("kappa", "core_a", "lia_only", "use_bh", "bh_quadtree", "bh_theta",
                     "bh_grain", "use_mf", "alpha", "alpha_p", "hyperfriction",
                     "max_curv_scale", "hyperalpha", "dl_max"):
            setattr(o, name, getattr(p, name))
        o.rk4_classic = 1 if rk4_classic else 0
        o.vn, o.vs, o.vb = _flow(p.vn), _flow(p.vs), _flow(p.vb)
        return o

    def update_tangle(self, t: HostTangle, p: Params, time=0.0) -> HostTangle:
        out = t.copy()
        ot, keep = self._tangle(t)
        op = self._params(p)
        self.lib.ovo_update_tangle(C.byref(ot), C.byref(op), C.c_double(time),
                                   out.dxi.ctypes.data_as(C.c_void_p), out.tangents.ctypes.data_as(C.c_void_p),
                                   out.normals.ctypes.data_as(C.c_void_p), out.vels.ctypes.data_as(C.c_void_p),
                                   out.vs.ctypes.data_as(C.c_void_p))
        return out

    def rk4_step(self, t: HostTangle, p: Params, time, dt, rk4_classic=False) -> HostTangle:
        """One step from t (whose vels must be current)."""
        out = t.copy()
        ot, keep = self._tangle(t)
        op = self._params(p, rk4_classic)
        self.lib.ovo_rk4_step(C.byref(ot), C.byref(op), C.c_double(time), C.c_double(dt),
                              out.pos.ctypes.data_as(C.c_void_p), t.vels.ctypes.data_as(C.c_void_p))
        return out

    def segments_at(self, t: HostTangle, p: Params, pts, skip=None) -> np.ndarray:
        pts = np.ascontiguousarray(pts, dtype=np.float64)
        out = np.zeros_like(pts)
        sk = None if skip is None else np.ascontiguousarray(skip, dtype=np.int32)
        ot, keep = self._tangle(t)
        op = self._params(p)
        self.lib.ovo_segments_at(C.byref(ot), C.byref(op), len(pts), C.c_void_p(pts.ctypes.data),
                                 None if sk is None else C.c_void_p(sk.ctypes.data),
                                 C.c_void_p(out.ctypes.data))
        return out

    def bh_at(self, t: HostTangle, p: Params, pts, skip=None) -> np.ndarray:
        pts = np.ascontiguousarray(pts, dtype=np.float64)
        out = np.zeros_like(pts)
        sk = None if skip is None else np.ascontiguousarray(skip, dtype=np.int32)
        ot, keep = self._tangle(t)
        op = self._params(p)
        self.lib.ovo_bh_at(C.byref(ot), C.byref(op), len(pts), C.c_void_p(pts.ctypes.data),
                           None if sk is None else C.c_void_p(sk.ctypes.data), C.c_void_p(out.ctypes.data))
        return out


# ---------------------------------------------------------------- reference
class Ref:
    """The reference's own functions on a HostTangle copy."""

    def __init__(self, path: Path = REF_SO, threads: int | None = None):
        if not Path(path).exists():
            raise FileNotFoundError(f"{path} not built (needs the reference sources)")
        self.lib = C.CDLL(str(path))
        self.lib.refh_set_flow.argtypes = [C.c_int, C.c_char_p, C.c_int, C.POINTER(C.c_char_p),
                                           C.POINTER(C.c_double)]
        for name in ("update_tangle", "refh_update_tangle", "refh_rk4_step",
                     "refh_update_velocities", "refh_update_tangents_normals"):
            if hasattr(self.lib, name):
                getattr(self.lib, name).restype = None
        self.lib.refh_calculate_vs.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        self.lib.refh_octree_vs.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_double,
                                            C.c_void_p]
        C.c_int.in_dll(self.lib, "global_num_threads").value = threads or os.cpu_count() or 1

    def configure(self, p: Params):
        p.apply_globals(self.lib)
        for which, f in enumerate((p.vn, p.vs, p.vb)):
            spec = FLOW_PARAMS[f.name]
            names = (C.c_char_p * max(1, len(spec)))(*[n.encode() for n, _ in spec])
            vals = (C.c_double * (3 * max(1, len(spec))))()
            for q, (n, ty) in enumerate(spec):
                v = f.params.get(n, 0.0)
                if ty == 2:
                    vals[3 * q:3 * q + 3] = [float(x) for x in v]
                else:
                    vals[3 * q] = float(v)
            rc = self.lib.refh_set_flow(which, f.name.encode(), len(spec), names, vals)
            assert rc == 0, f.name

    def _copy(self, t: HostTangle) -> HostTangle:
        out = t.copy()
        out.set_images_from_library(self.lib)
        return out

    def update_tangle(self, t: HostTangle, p: Params, time=0.0) -> HostTangle:
        self.configure(p)
        out = self._copy(t)
        self.lib.refh_update_tangle(out.ptr(), C.c_double(time))
        return out

    def update_velocities(self, t: HostTangle, p: Params, time=0.0) -> HostTangle:
        self.configure(p)
        out = self._copy(t)
        self.lib.refh_update_velocities(out.ptr(), C.c_double(time))
        return out

    def rk4_step(self, t: HostTangle, p: Params, time, dt) -> HostTangle:
        self.configure(p)
        out = self._copy(t)
        self.lib.refh_rk4_step(out.ptr(), C.c_double(time), C.c_double(dt))
        return out

    def update_tangents_normals(self, t: HostTangle, p: Params) -> HostTangle:
        """The reference's update_tangents_normals (src/tangle.c:704-727) on a copy."""
        self.configure(p)
        out = self._copy(t)
        f = self.lib.update_tangents_normals
        f.restype = None
        f.argtypes = [C.c_void_p]
        f(C.cast(out.ptr(), C.c_void_p))
        return out

    def remesh(self, t: HostTangle, p: Params, min_dist, max_dist) -> HostTangle:
        """The reference's remesh (src/tangle.c:824-873) on a copy whose dxi,
        tangents and normals are current; the copy keeps t's next_free."""
        self.configure(p)
        out = self._copy(t)
        out.struct.next_free = t.struct.next_free
        f = self.lib.remesh
        f.restype = None
        f.argtypes = [C.c_void_p, C.c_double, C.c_double]
        f(C.cast(out.ptr(), C.c_void_p), min_dist, max_dist)
        return out

    def eliminate_small_loops(self, t: HostTangle, p: Params, loop_length: int) -> HostTangle:
        """The reference's eliminate_small_loops (src/tangle.c:876-943) on a
        copy, with the loop-removal globals as they are set in its library."""
        self.configure(p)
        out = self._copy(t)
        f = self.lib.eliminate_small_loops
        f.restype = None
        f.argtypes = [C.c_void_p, C.c_int]
        f(C.cast(out.ptr(), C.c_void_p), loop_length)
        return out

    def enforce_boundaries(self, t: HostTangle, p: Params) -> HostTangle:
        """The reference's enforce_boundaries (src/tangle.c:796-819) on a copy."""
        self.configure(p)
        out = self._copy(t)
        f = self.lib.enforce_boundaries
        f.restype = None
        f.argtypes = [C.c_void_p]
        f(C.cast(out.ptr(), C.c_void_p))
        return out

    def reconnect(self, t: HostTangle, p: Params, time, rec_dist, rec_angle):
        """The reference's reconnect (src/vortex_dynamics.c:140-313) on a copy
        whose tangents and normals are current; returns (copy, count)."""
        self.configure(p)
        out = self._copy(t)
        f = self.lib.reconnect
        f.restype = C.c_int
        f.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double]
        n = f(C.cast(out.ptr(), C.c_void_p), time, rec_dist, rec_angle)
        return out, n

    def segments_at(self, t: HostTangle, p: Params, pts, skip=None) -> np.ndarray:
        self.configure(p)
        tt = self._copy(t)
        pts = np.ascontiguousarray(pts, dtype=np.float64)
        out = np.zeros_like(pts)
        sk = None if skip is None else np.ascontiguousarray(skip, dtype=np.int32)
        self.lib.refh_calculate_vs(C.cast(tt.ptr(), C.c_void_p), len(pts), pts.ctypes.data,
                                   None if sk is None else sk.ctypes.data, out.ctypes.data)
        return out

    def bh_at(self, t: HostTangle, p: Params, pts, skip=None) -> np.ndarray:
        self.configure(p)
        tt = self._copy(t)
        pts = np.ascontiguousarray(pts, dtype=np.float64)
        out = np.zeros_like(pts)
        sk = None if skip is None else np.ascontiguousarray(skip, dtype=np.int32)
        self.lib.refh_octree_vs(C.cast(tt.ptr(), C.c_void_p), len(pts), pts.ctypes.data,
                                None if sk is None else sk.ctypes.data, C.c_double(p.bh_theta),
                                out.ctypes.data)
        return out


def have_ref() -> bool:
    return REF_SO.exists()


def rel_err(a: np.ndarray, b: np.ndarray, mask=None) -> float:
    """max over nodes of |a - b| / |b| (per-node vector norms)."""
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
