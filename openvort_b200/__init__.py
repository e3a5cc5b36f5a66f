"""openvort_b200: OpenVort's Schwarz vortex-filament velocity + RK4 path on
NVIDIA B200 (sm_100a).

The compute lives in libov_gpu.so (CUDA, C ABI in include/openvort_b200.h);
this package is the Python host side: the ctypes mirror of the reference's
tangle structures and globals (`tangle`), seeded workload generators
(`geometry`), and thin wrappers that call the library and raise on errors.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import (OV_FIELD_ALL, OV_FIELD_DXI, OV_FIELD_NORMALS, OV_FIELD_POS, OV_FIELD_TANGENTS, OV_FIELD_VELS,
                   OV_FIELD_VS, OV_PREC_FP64, OV_PREC_MIXED, OVError, check, load, stats)
from .tangle import EMPTY, FREE, PINNED, PINNED_SLIP, Flow, HostTangle, Params

__all__ = [
    "OVError", "Params", "Flow", "HostTangle", "DeviceState", "load", "configure",
    "update_tangle", "update_velocities", "update_tangents_normals", "rk4_step", "euler_step",
    "set_precision", "OV_PREC_FP64", "OV_PREC_MIXED",
]


def configure(params: Params, precision: int = OV_PREC_FP64, rk4_classic: bool = False):
    """Write the hot-path globals and flows into libov_gpu.so."""
    lib = load()
    params.apply_globals(lib)
    params.apply_flows(lib)
    lib.ov_set_precision(precision)
    lib.ov_set_rk4_classic(1 if rk4_classic else 0)
    return lib


def set_precision(mode: int):
    load().ov_set_precision(mode)


def _prep(t: HostTangle):
    lib = load()
    t.set_images_from_library(lib)
    return lib


def update_tangents_normals(t: HostTangle):
    lib = _prep(t)
    lib.update_tangents_normals(t.ptr())
    check(lib)


def update_velocities(t: HostTangle, time: float = 0.0):
    lib = _prep(t)
    lib.update_velocities(t.ptr(), time, None)
    check(lib)


def update_tangle(t: HostTangle, time: float = 0.0):
    """update_tangents_normals + update_velocities (include/tangle.h:160-164)."""
    update_tangents_normals(t)
    update_velocities(t, time)


def rk4_step(t: HostTangle, time: float, dt: float):
    lib = _prep(t)
    lib.rk4_step(t.ptr(), time, dt)
    check(lib)


def euler_step(t: HostTangle, dt: float):
    lib = _prep(t)
    lib.euler_step(t.ptr(), dt)
    check(lib)


class DeviceState:
    """A tangle resident in device memory for multi-step runs (ov_state_*)."""

    def __init__(self, t: HostTangle):
        self.lib = _prep(t)
        self.h = self.lib.ov_state_create()
        check(self.lib)
        if not self.h:
            raise OVError(1, "ov_state_create failed")
        self.t = t
        self._rc(self.lib.ov_state_upload(self.h, t.ptr()))

    def _rc(self, rc):
        if rc != 0:
            check(self.lib)
            raise OVError(rc, "call failed")

    def update_tangle(self, time: float):
        self._rc(self.lib.ov_state_update_tangle(self.h, time))

    def rk4_step(self, time: float, dt: float):
        self._rc(self.lib.ov_state_rk4_step(self.h, time, dt))

    def run(self, t0: float, dt: float, nsteps: int):
        self._rc(self.lib.ov_state_run(self.h, t0, dt, nsteps))

    def download(self, what: int = OV_FIELD_ALL):
        self._rc(self.lib.ov_state_download(self.h, self.t.ptr(), what))

    def upload(self):
        """Copy the host tangle (positions, links, status, vels) in again."""
        self._rc(self.lib.ov_state_upload(self.h, self.t.ptr()))

    # one tangle over several ranks (ov_state_shard*); openvort_b200.shard
    # drives these with the exchange between begin and end
    def shard_bytes(self, world: int) -> int:
        return int(self.lib.ov_state_shard_bytes(self.h, world))

    def shard(self, rank: int, world: int, xbuf_ptr: int | None, nbytes: int = 0):
        self._rc(self.lib.ov_state_shard(self.h, rank, world, xbuf_ptr, nbytes))

    def shard_begin(self, stage: int, time: float, dt: float):
        self._rc(self.lib.ov_state_shard_begin(self.h, stage, time, dt))

    def shard_end(self, stage: int, time: float, dt: float):
        self._rc(self.lib.ov_state_shard_end(self.h, stage, time, dt))

    def save_frame(self, path: str, time: float, binary: bool = True):
        """Start writing a frame of the current state (ov_state_save_frame);
        wait_frames() waits for the file."""
        fmt = _lib.OV_FRAME_BINARY if binary else _lib.OV_FRAME_TEXT
        self._rc(self.lib.ov_state_save_frame(self.h, str(path).encode(), time, fmt))

    def wait_frames(self):
        self._rc(self.lib.ov_frame_wait())

    def eval_points(self, pts: np.ndarray, skip=None, method: int = 0) -> np.ndarray:
        pts = np.ascontiguousarray(pts, dtype=np.float64)
        out = np.zeros_like(pts)
        sk = None if skip is None else np.ascontiguousarray(skip, dtype=np.int32)
        self._rc(self.lib.ov_state_eval_points(
            self.h, len(pts), pts.ctypes.data, None if sk is None else sk.ctypes.data, method,
            out.ctypes.data))
        return out

    def stats(self) -> "_lib.RunStats":
        s = _lib.RunStats()
        self._rc(self.lib.ov_state_get_stats(self.h, C.byref(s)))
        return s

    def reset_stats(self):
        self.lib.ov_state_reset_stats(self.h)

    def close(self):
        if self.h:
            self.lib.ov_state_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceBatch:
    """An ensemble of independent open-boundary systems resident in device
    memory (ov_batch_*): system s occupies slots offsets[s] .. offsets[s+1]-1
    of the one HostTangle `t`."""

    def __init__(self, t: HostTangle, offsets):
        self.lib = load()
        self.t = t
        self.offsets = np.ascontiguousarray(offsets, dtype=np.int32)
        self.h = self.lib.ov_batch_create(t.ptr(), len(self.offsets) - 1, self.offsets.ctypes.data)
        if not self.h:
            check(self.lib)
            raise OVError(1, "ov_batch_create failed")

    def _rc(self, rc):
        if rc != 0:
            check(self.lib)
            raise OVError(rc, "call failed")

    def update(self, time: float = 0.0):
        self._rc(self.lib.ov_batch_update(self.h, time))

    def run(self, t0: float, dt: float, nsteps: int):
        self._rc(self.lib.ov_batch_run(self.h, t0, dt, nsteps))

    def download(self, what: int = OV_FIELD_ALL):
        self._rc(self.lib.ov_batch_download(self.h, self.t.ptr(), what))

    def tuning(self) -> "_lib.BatchTuning":
        tu = _lib.BatchTuning()
        self._rc(self.lib.ov_batch_get_tuning(self.h, C.byref(tu)))
        return tu

    def set_tuning(self, targets_per_block: int, sources_per_tile: int, blocks_per_sm: int = 0):
        tu = _lib.BatchTuning(targets_per_block, sources_per_tile, blocks_per_sm, 0.0)
        self._rc(self.lib.ov_batch_set_tuning(self.h, C.byref(tu)))

    def autotune(self) -> "_lib.BatchTuning":
        tu = _lib.BatchTuning()
        self._rc(self.lib.ov_batch_autotune(self.h, C.byref(tu)))
        return tu

    def stats(self) -> "_lib.BatchStats":
        s = _lib.BatchStats()
        self._rc(self.lib.ov_batch_get_stats(self.h, C.byref(s)))
        return s

    def close(self):
        if self.h:
            self.lib.ov_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
