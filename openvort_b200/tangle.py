"""Host-side mirror of OpenVort's tangle structures and run-time globals.

`TangleState` has the byte layout of the reference's `struct tangle_state`
(include/tangle.h:82-106 of the reference), so one numpy-backed tangle can be
handed to libov_gpu.so's reference-named entry points (update_velocities,
rk4_step, ...) or to any other library with the same ABI.  `Params` holds the
globals those entry points read (include/vortex_constants.h:25-78) and the
external-flow configurations (include/external_velocity.h:80-90) and writes
them into a loaded library.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Dict, Optional, Sequence, Tuple

import numpy as np

# node status (include/tangle.h:28-33)
EMPTY, FREE, PINNED, PINNED_SLIP = -1, 0, 1, 2
# wall types (include/vec3_maths.h:31) and faces (:39-44)
WALL_OPEN, WALL_PERIODIC, WALL_MIRROR = 0, 1, 2
X_L, X_H, Y_L, Y_H, Z_L, Z_H = range(6)


class Vec3d(C.Structure):
    _fields_ = [("p", C.c_double * 3)]


class DomainBox(C.Structure):
    _fields_ = [("bottom_left_back", Vec3d), ("top_right_front", Vec3d), ("wall", C.c_int * 6)]


class ImageTangle(C.Structure):
    _fields_ = [("shift", C.c_int * 3), ("reflect", C.c_int)]


class BoundaryImages(C.Structure):
    _fields_ = [("images", C.POINTER(ImageTangle)), ("n", C.c_int)]


class NodeStatus(C.Structure):
    _fields_ = [("status", C.c_int), ("pin_wall", C.c_int)]


class Neighbour(C.Structure):
    _fields_ = [("forward", C.c_int), ("reverse", C.c_int)]


class TangleState(C.Structure):
    _fields_ = [
        ("vnodes", C.POINTER(Vec3d)),
        ("vnodes_new", C.POINTER(Vec3d)),
        ("vels", C.POINTER(Vec3d)),
        ("vs", C.POINTER(Vec3d)),
        ("tangents", C.POINTER(Vec3d)),
        ("normals", C.POINTER(Vec3d)),
        ("dxi", C.POINTER(C.c_double)),
        ("recalculate", C.POINTER(C.c_int)),
        ("connections", C.POINTER(Neighbour)),
        ("status", C.POINTER(NodeStatus)),
        ("box", DomainBox),
        ("bimg", BoundaryImages),
        ("N", C.c_int),
        ("next_free", C.c_int),
        ("total_free", C.c_int),
    ]


class _ParamValue(C.Union):
    _fields_ = [("vector", Vec3d), ("scalar", C.c_double)]


class VParam(C.Structure):
    _fields_ = [("name", C.c_char_p), ("type", C.c_int), ("value", _ParamValue)]


class VConf(C.Structure):
    _fields_ = [("name", C.c_char_p), ("fun", C.c_void_p), ("n_params", C.c_int),
                ("v_params", VParam * 32)]


SCALAR_PARAM, VECTOR_PARAM = 1, 2

# Boundary-image tables: shift (x, y, z) and mirror face (-1 none), in the
# reference's order (src/boundary_images.c:26-163).  Used where a tangle's
# image table must be built on the Python side (the libraries export theirs).
_P26 = [(a, b, c) for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1) if (a, b, c) != (0, 0, 0)]
IMAGE_TABLES: Dict[str, list] = {
    "open": [],
    "periodic-6": [(s, -1) for s in _P26 if sum(map(abs, s)) == 1],
    "periodic-18": [(s, -1) for s in _P26 if sum(map(abs, s)) <= 2],
    "periodic-26": [(s, -1) for s in _P26],
    "periodic-z-open-xy": [((0, 0, -1), -1), ((0, 0, 1), -1)],
    "wall-1-open": [((0, 0, -1), Z_L)],
}
# wall settings per boundary name (src/configuration.c:333-392)
BOUNDARY_WALLS = {
    "open": [WALL_OPEN] * 6,
    "periodic-6": [WALL_PERIODIC] * 6,
    "periodic-18": [WALL_PERIODIC] * 6,
    "periodic-26": [WALL_PERIODIC] * 6,
    "periodic-z-open-xy": [WALL_OPEN] * 4 + [WALL_PERIODIC] * 2,
    "wall-1-open": [WALL_OPEN] * 4 + [WALL_MIRROR, WALL_OPEN],
}
# exported table symbol per boundary name (include/tangle.h:62-77)
BOUNDARY_SYMBOLS = {
    "open": "open_boundaries", "periodic-6": "periodic_6", "periodic-18": "periodic_18",
    "periodic-26": "periodic_26", "periodic-z-open-xy": "periodic_z_open_xy",
    "wall-1-open": "wall_1_open", "wall-1-18": "wall_1_18", "wall-1-26": "wall_1_26",
    "wall-2-4": "wall_2_4", "wall-2-2": "wall_2_2", "wall-2-26": "wall_2_26",
    "channel-z": "channel_z",
}


class HostTangle:
    """A tangle whose arrays live in numpy buffers (optionally pinned host
    memory) and whose `struct tangle_state` points at them."""

    def __init__(self, pos: np.ndarray, fwd: np.ndarray, rev: np.ndarray,
                 status: Optional[np.ndarray] = None, pin_wall: Optional[np.ndarray] = None,
                 box_lo=(0.0, 0.0, 0.0), box_hi=(1.0, 1.0, 1.0), boundary: str = "open",
                 alloc=np.empty):
        n = int(pos.shape[0])
        self.n = n
        self.boundary = boundary

        def buf(shape, dtype):
            a = alloc(shape, dtype=dtype)
            a[...] = 0
            return a

        self.pos = buf((n, 3), np.float64)
        self.pos[:] = pos
        self.pos_new = buf((n, 3), np.float64)
        self.vels = buf((n, 3), np.float64)
        self.vs = buf((n, 3), np.float64)
        self.tangents = buf((n, 3), np.float64)
        self.normals = buf((n, 3), np.float64)
        self.dxi = buf((n,), np.float64)
        self.recalc = buf((n,), np.int32)
        self.links = buf((n, 2), np.int32)
        self.links[:, 0] = fwd
        self.links[:, 1] = rev
        self.stat = buf((n, 2), np.int32)
        self.stat[:, 0] = FREE if status is None else status
        self.stat[:, 1] = -1 if pin_wall is None else pin_wall
        self.box_lo = tuple(float(x) for x in box_lo)
        self.box_hi = tuple(float(x) for x in box_hi)
        self.walls = list(BOUNDARY_WALLS.get(boundary, [WALL_OPEN] * 6))
        self.struct = TangleState()
        self._bimg_keep = None
        self._bind()

    def _bind(self):
        s = self.struct

        def vp(a):
            return a.ctypes.data_as(C.POINTER(Vec3d))

        s.vnodes = vp(self.pos)
        s.vnodes_new = vp(self.pos_new)
        s.vels = vp(self.vels)
        s.vs = vp(self.vs)
        s.tangents = vp(self.tangents)
        s.normals = vp(self.normals)
        s.dxi = self.dxi.ctypes.data_as(C.POINTER(C.c_double))
        s.recalculate = self.recalc.ctypes.data_as(C.POINTER(C.c_int))
        s.connections = self.links.ctypes.data_as(C.POINTER(Neighbour))
        s.status = self.stat.ctypes.data_as(C.POINTER(NodeStatus))
        for c in range(3):
            s.box.bottom_left_back.p[c] = self.box_lo[c]
            s.box.top_right_front.p[c] = self.box_hi[c]
        for f in range(6):
            s.box.wall[f] = self.walls[f]
        s.N = self.n
        s.next_free = 0
        s.total_free = 0
        self.set_images_from_table(IMAGE_TABLES.get(self.boundary, []))

    def set_images_from_table(self, table):
        arr = (ImageTangle * max(1, len(table)))()
        for j, (sh, refl) in enumerate(table):
            arr[j].shift[:] = list(sh)
            arr[j].reflect = refl
        self._bimg_keep = arr
        self.struct.bimg.images = C.cast(arr, C.POINTER(ImageTangle)) if table else None
        self.struct.bimg.n = len(table)

    def set_images_from_library(self, lib: C.CDLL):
        """Point bimg at the boundary table exported by `lib`."""
        sym = BOUNDARY_SYMBOLS[self.boundary]
        self.struct.bimg = BoundaryImages.in_dll(lib, sym)
        self._bimg_keep = None

    def ptr(self):
        return C.byref(self.struct)

    @property
    def active(self) -> np.ndarray:
        return self.stat[:, 0] != EMPTY

    def copy(self, alloc=np.empty) -> "HostTangle":
        t = HostTangle(self.pos, self.links[:, 0], self.links[:, 1], self.stat[:, 0],
                       self.stat[:, 1], self.box_lo, self.box_hi, self.boundary, alloc=alloc)
        for name in ("vels", "vs", "tangents", "normals", "dxi"):
            getattr(t, name)[:] = getattr(self, name)
        return t


# parameter names per flow in the reference's v_confs[] (src/external_velocity.c:85-170)
FLOW_PARAMS = {
    "no flow": [],
    "spherical": [("strength", SCALAR_PARAM), ("cutoff", SCALAR_PARAM)],
    "simple": [("external_v", VECTOR_PARAM)],
    "spherical and simple": [("external_v", VECTOR_PARAM), ("strength", SCALAR_PARAM),
                             ("cutoff", SCALAR_PARAM)],
    "cylindrical": [("strength", SCALAR_PARAM), ("cutoff", SCALAR_PARAM)],
    "oscillating": [("strength", SCALAR_PARAM), ("frequency", SCALAR_PARAM),
                    ("wave", VECTOR_PARAM), ("polarization", VECTOR_PARAM)],
    "oscillating slit": [("strength", SCALAR_PARAM), ("frequency", SCALAR_PARAM),
                         ("cutoff", SCALAR_PARAM)],
    "coscos": [("k", SCALAR_PARAM), ("v0", SCALAR_PARAM), ("l", SCALAR_PARAM)],
    "coscos-divfree": [("k", SCALAR_PARAM), ("v0", SCALAR_PARAM), ("l", SCALAR_PARAM)],
    "cos-divfree": [("k", SCALAR_PARAM), ("v0", SCALAR_PARAM), ("l", SCALAR_PARAM)],
    "simple-shear": [("rate", SCALAR_PARAM), ("v0", SCALAR_PARAM)],
    "rotosc": [("freq", SCALAR_PARAM), ("amp", SCALAR_PARAM)],
    "DG": [("rot", SCALAR_PARAM), ("vz", SCALAR_PARAM)],
    "rotosc-boundary": [("freq", SCALAR_PARAM), ("amp", SCALAR_PARAM)],
    "constant acceleration": [("accel", SCALAR_PARAM)],
    "parabolic": [("H", SCALAR_PARAM), ("amp", SCALAR_PARAM)],
}
FLOW_KINDS = list(FLOW_PARAMS.keys())


@dataclass
class Flow:
    name: str = "no flow"
    params: Dict[str, object] = field(default_factory=dict)

    def vconf(self) -> Tuple[VConf, list]:
        """A struct v_conf_t with this flow's name and parameters (fun NULL)."""
        spec = FLOW_PARAMS[self.name]
        c = VConf()
        keep = [self.name.encode()]
        c.name = keep[0]
        c.fun = None
        c.n_params = len(spec)
        for q, (pname, ptype) in enumerate(spec):
            b = pname.encode()
            keep.append(b)
            c.v_params[q].name = b
            c.v_params[q].type = ptype
            val = self.params.get(pname, 0.0)
            if ptype == VECTOR_PARAM:
                c.v_params[q].value.vector.p[:] = [float(x) for x in val]
            else:
                c.v_params[q].value.scalar = float(val)
        return c, keep


@dataclass
class Params:
    """The reference's run-time globals for the hot path, with its defaults
    (src/vortex_constants.c:24-95)."""
    kappa: float = 9.97e-4
    core_a: float = 1e-8
    lia_only: int = 0
    use_bh: int = 0
    bh_theta: float = 0.1
    bh_quadtree: int = 0
    bh_grain: float = 1e-8
    use_mf: int = 1
    alpha: float = 0.1
    alpha_p: float = 0.01
    hyperfriction: int = 1
    max_curv_scale: float = 0.2
    hyperalpha: float = 0.5
    dl_max: float = 5e-3
    vn: Flow = field(default_factory=Flow)
    vs: Flow = field(default_factory=Flow)
    vb: Flow = field(default_factory=Flow)

    GLOBALS = [("KAPPA", "kappa", C.c_double), ("VORTEX_WIDTH", "core_a", C.c_double),
               ("global_LIA_only", "lia_only", C.c_int), ("global_use_BH", "use_bh", C.c_int),
               ("global_BH_resolution", "bh_theta", C.c_double),
               ("global_BH_quadtree", "bh_quadtree", C.c_int),
               ("global_BH_grain", "bh_grain", C.c_double),
               ("global_use_mutual_friction", "use_mf", C.c_int),
               ("global_alpha", "alpha", C.c_double), ("global_alpha_p", "alpha_p", C.c_double),
               ("global_hyperfriction", "hyperfriction", C.c_int),
               ("global_max_curvature_scale", "max_curv_scale", C.c_double),
               ("global_hyperalpha", "hyperalpha", C.c_double),
               ("global_dl_max", "dl_max", C.c_double)]

    def apply_globals(self, lib: C.CDLL):
        for sym, attr, ctype in self.GLOBALS:
            ctype.in_dll(lib, sym).value = getattr(self, attr)

    def apply_flows(self, lib: C.CDLL):
        """Write vn_conf / vs_conf / vb_conf by name (fun left NULL).  The
        name strings stay referenced from the library handle."""
        keepall = []
        for sym, flow in (("vn_conf", self.vn), ("vs_conf", self.vs), ("vb_conf", self.vb)):
            conf, keep = flow.vconf()
            keepall.append((conf, keep))
            C.memmove(C.addressof(VConf.in_dll(lib, sym)), C.addressof(conf), C.sizeof(VConf))
        lib._ov_flow_strings = keepall


def perpendicular(d: Sequence[float]) -> np.ndarray:
    """A unit vector normal to d (perpendicular, src/vortex_utils.c:29-46)."""
    d = np.asarray(d, dtype=np.float64)
    for a in (np.array([1.0, 0, 0]), np.array([0, 1.0, 0])):
        res = d * (-(a @ d)) + a
        nr = np.sqrt(res @ res)
        if nr > 1e-8 or a[1] == 1.0:
            return res * (1 / nr)
    raise AssertionError


def ring_points(center, direction, radius: float, n: int) -> np.ndarray:
    """Points of a circle as add_circle places them (src/vortex_utils.c:52-99):
    basis u = perp x dir, v = dir x u, point k at angle 2 pi k / n."""
    d = np.asarray(direction, dtype=np.float64)
    z = perpendicular(d)
    u = np.cross(z, d)
    v = np.cross(d, u)
    u = u * (1 / np.sqrt(u @ u))
    v = v * (1 / np.sqrt(v @ v))
    k = np.arange(n, dtype=np.float64)
    phi = 2 * np.pi / n * k
    return (u[None, :] * (radius * np.cos(phi))[:, None] + v[None, :] * (radius * np.sin(phi))[:, None]
            + np.asarray(center, dtype=np.float64)[None, :])
