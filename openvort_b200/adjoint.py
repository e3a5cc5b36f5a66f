"""Gradients through the vortex-filament dynamics (ov_adjoint_*).

`Adjoint` wraps one tangle of closed loops in open space; `trajectory` runs
nsteps RK4 steps of it as a `torch.autograd.Function`, so a loss written in
torch on the final positions back-propagates to the initial positions and to
the normal-fluid velocity vector vn (the "simple" flow driving mutual
friction).  The reverse sweep is the library's own: positions are
checkpointed every `every` steps and each block of steps is recomputed from
its checkpoint before it is run backwards.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import OVError, check, load
from .tangle import HostTangle


def _arr(x, n=None) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float64))
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


class Adjoint:
    """Forward and reverse sweeps of one tangle (its topology is fixed)."""

    def __init__(self, t: HostTangle):
        self.lib = load()
        self.t = t
        self.n = t.n
        self.h = self.lib.ov_adjoint_create(t.ptr())
        if not self.h:
            check(self.lib)
            raise OVError(1, "ov_adjoint_create failed")

    def _rc(self, rc):
        if rc != 0:
            check(self.lib)
            raise OVError(rc, "call failed")

    def _vn(self, vn):
        return None if vn is None else _arr(vn, 3)

    def velocity(self, x, vn=None, t: float = 0.0) -> np.ndarray:
        x = _arr(x, 3 * self.n)
        v = np.zeros((self.n, 3))
        vv = self._vn(vn)
        self._rc(self.lib.ov_adjoint_velocity(self.h, x.ctypes.data, None if vv is None else vv.ctypes.data,
                                              t, v.ctypes.data))
        return v

    def velocity_vjp(self, x, v_bar, vn=None, t: float = 0.0):
        x = _arr(x, 3 * self.n)
        g = _arr(v_bar, 3 * self.n)
        xb = np.zeros((self.n, 3))
        vnb = np.zeros(3)
        vv = self._vn(vn)
        self._rc(self.lib.ov_adjoint_velocity_vjp(self.h, x.ctypes.data,
                                                  None if vv is None else vv.ctypes.data, t, g.ctypes.data,
                                                  xb.ctypes.data, vnb.ctypes.data))
        return xb, vnb

    def forward(self, x0, vn, t0: float, dt: float, nsteps: int, every: int = 32) -> np.ndarray:
        x0 = _arr(x0, 3 * self.n)
        out = np.zeros((self.n, 3))
        vv = self._vn(vn)
        self._rc(self.lib.ov_adjoint_forward(self.h, x0.ctypes.data, None if vv is None else vv.ctypes.data,
                                             t0, dt, nsteps, every, out.ctypes.data))
        return out

    @property
    def generation(self) -> int:
        """Completed forward runs; backward refers to the last one."""
        return int(self.lib.ov_adjoint_generation(self.h))

    def backward(self, x_final_bar):
        g = _arr(x_final_bar, 3 * self.n)
        xb = np.zeros((self.n, 3))
        vnb = np.zeros(3)
        self._rc(self.lib.ov_adjoint_backward(self.h, g.ctypes.data, xb.ctypes.data, vnb.ctypes.data))
        return xb, vnb

    def close(self):
        if self.h:
            self.lib.ov_adjoint_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _function():
    import torch

    class RK4Trajectory(torch.autograd.Function):
        """x_final = RK4^nsteps(x0; vn); backward through ov_adjoint_backward."""

        @staticmethod
        def forward(ctx, x0, vn, adj, t0, dt, nsteps, every):
            args = (x0.detach().cpu().numpy().copy(), vn.detach().cpu().numpy().copy(), t0, dt, nsteps, every)
            xf = adj.forward(*args)
            ctx.adj = adj
            ctx.args = args
            ctx.generation = adj.generation
            ctx.dev = (x0.device, vn.device)
            return torch.from_numpy(xf).to(x0.device)

        @staticmethod
        def backward(ctx, g):
            # another trajectory on the same handle since this one: its
            # checkpoints are gone, so run this forward again first
            if ctx.adj.generation != ctx.generation:
                ctx.adj.forward(*ctx.args)
                ctx.generation = ctx.adj.generation
            xb, vnb = ctx.adj.backward(g.detach().cpu().numpy())
            return (torch.from_numpy(xb).to(ctx.dev[0]), torch.from_numpy(vnb).to(ctx.dev[1]),
                    None, None, None, None, None)

    return RK4Trajectory


_RK4 = None


def trajectory(adj: Adjoint, x0, vn, t0: float, dt: float, nsteps: int, every: int = 32):
    """Differentiable final positions (torch tensors of float64: x0 (N, 3),
    vn (3,))."""
    global _RK4
    if _RK4 is None:
        _RK4 = _function()
    return _RK4.apply(x0, vn, adj, t0, dt, nsteps, every)


def centroid_length_loss(x, fwd: np.ndarray, active: np.ndarray, target):
    """|centroid - target|^2 + total line length, for torch positions x:
    the centroid is the mean of the active nodes, the length the sum of the
    segments x_k -> x_fwd(k)."""
    import torch
    idx = torch.as_tensor(np.nonzero(active)[0], device=x.device)
    nxt = torch.as_tensor(np.asarray(fwd)[np.nonzero(active)[0]], device=x.device, dtype=torch.long)
    c = x[idx].mean(dim=0)
    tgt = torch.as_tensor(np.asarray(target, dtype=np.float64), device=x.device)
    seg = x[nxt] - x[idx]
    return ((c - tgt) ** 2).sum() + torch.sqrt((seg * seg).sum(dim=1)).sum()
