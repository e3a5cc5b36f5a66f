"""GPU: reverse-mode derivatives (ov_adjoint_*, openvort_b200.adjoint).

Each gradient is checked against FP64 central finite differences of the
forward computation of the same library:
  - the velocity's vector-Jacobian product, along a random direction of the
    positions and along the normal-fluid vector: relative error <= 1e-6;
  - the gradient of |centroid - target|^2 + line length after 20 RK4 steps
    of a ring with Kelvin waves, through the torch.autograd.Function, with
    respect to the initial positions and vn: <= 1e-6 with the FP64 forward
    and with the mixed one (two-float offsets in slot order at this size);
  - the checkpoint interval changes nothing (1e-13).
"""
import numpy as np
import pytest

from openvort_b200 import geometry as G
from openvort_b200.tangle import Flow, Params

pytestmark = pytest.mark.gpu

N = 128
R0 = 1e-2
DL = 2 * np.pi * R0 / N
# Hyperfriction switches on where the curvature exceeds max_curv_scale /
# dl_max, so the dynamics are only piecewise smooth: dl_max = DL/4 puts that
# threshold (1600 /cm) far above the ring's curvature (<= ~360 /cm), so no
# node crosses it between the perturbed runs of the finite differences.
# The branch itself is checked with hyperfriction active at every node.
PARAMS = Params(kappa=9.97e-4, core_a=1e-8, use_mf=1, alpha=0.098, alpha_p=0.016, hyperfriction=1,
                max_curv_scale=0.2, hyperalpha=0.5, dl_max=DL / 4,
                vn=Flow("simple", {"external_v": (0.2, 0.0, 0.0)}), vs=Flow("no flow"))
VN = np.array([0.2, 0.0, 0.0])
DT, STEPS = 1e-5, 20       # omega dt ~ 0.3 for the grid-scale Kelvin waves
TARGET = np.array([0.004, -0.002, 0.003])


@pytest.fixture(scope="module")
def ov():
    import openvort_b200 as ov
    lib = ov.load()
    assert lib.ov_init(0) == 0, lib.ov_last_error_message()
    return ov


def kelvin_tangle():
    pos = G.kelvin_ring(11, n=N, radius=R0, modes=(2, 16), sigma=1e-4)
    return G.rings_to_tangle([pos], (-0.05,) * 3, (0.05,) * 3, "open")


@pytest.fixture
def adj(ov):
    from openvort_b200.adjoint import Adjoint
    ov.configure(PARAMS, ov.OV_PREC_FP64)
    t = kelvin_tangle()
    a = Adjoint(t)
    yield t, a
    a.close()
    ov.configure(PARAMS, ov.OV_PREC_FP64)


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def test_adjoint_velocity_matches_update_tangle(ov, adj):
    t, a = adj
    ref = t.copy()
    ov.update_tangle(ref, 0.0)
    v = a.velocity(t.pos, VN)
    assert np.max(np.linalg.norm(v - ref.vels, axis=1) / np.linalg.norm(ref.vels, axis=1)) < 1e-13


def test_velocity_vjp_with_hyperfriction_everywhere(ov):
    """dl_max = 10 DL: threshold 20 /cm below every node's curvature."""
    import dataclasses
    from openvort_b200.adjoint import Adjoint
    ov.configure(dataclasses.replace(PARAMS, dl_max=10 * DL), ov.OV_PREC_FP64)
    t = kelvin_tangle()
    a = Adjoint(t)
    rng = np.random.default_rng(6)
    g = rng.normal(size=(N, 3))
    d = rng.normal(size=(N, 3)) * DL
    xb, _ = a.velocity_vjp(t.pos, g, VN)
    eps = 1e-5
    fd = np.sum(g * (a.velocity(t.pos + eps * d, VN) - a.velocity(t.pos - eps * d, VN))) / (2 * eps)
    assert rel(np.sum(xb * d), fd) < 1e-6
    a.close()
    ov.configure(PARAMS, ov.OV_PREC_FP64)


def test_velocity_vjp_matches_central_differences(adj):
    t, a = adj
    rng = np.random.default_rng(5)
    g = rng.normal(size=(N, 3))
    d = rng.normal(size=(N, 3)) * DL
    xb, vnb = a.velocity_vjp(t.pos, g, VN)
    eps = 1e-5
    fd = np.sum(g * (a.velocity(t.pos + eps * d, VN) - a.velocity(t.pos - eps * d, VN))) / (2 * eps)
    assert rel(np.sum(xb * d), fd) < 1e-6
    ev = 1e-3
    for c in range(3):
        e = np.zeros(3)
        e[c] = ev
        fdv = np.sum(g * (a.velocity(t.pos, VN + e) - a.velocity(t.pos, VN - e))) / (2 * ev)
        assert abs(vnb[c] - fdv) <= 1e-6 * max(abs(fdv), np.max(np.abs(vnb)))


def _loss_value(a, t, x0, vn):
    import torch
    from openvort_b200.adjoint import centroid_length_loss
    xf = a.forward(x0, vn, 0.0, DT, STEPS, 8)
    return float(centroid_length_loss(torch.from_numpy(xf), t.links[:, 0], t.active, TARGET))


def _grads(a, t, every):
    import torch
    from openvort_b200.adjoint import centroid_length_loss, trajectory
    x0 = torch.tensor(t.pos, dtype=torch.float64, requires_grad=True)
    vn = torch.tensor(VN, dtype=torch.float64, requires_grad=True)
    xf = trajectory(a, x0, vn, 0.0, DT, STEPS, every)
    loss = centroid_length_loss(xf, t.links[:, 0], t.active, TARGET)
    loss.backward()
    return x0.grad.numpy().copy(), vn.grad.numpy().copy()


@pytest.mark.parametrize("precision,tol", [(0, 1e-6), (1, 1e-6)])
def test_trajectory_gradient_matches_central_differences(ov, adj, precision, tol):
    t, a = adj
    ov.configure(PARAMS, precision)
    gx, gv = _grads(a, t, every=8)
    ov.configure(PARAMS, ov.OV_PREC_FP64)   # finite differences of the FP64 dynamics
    rng = np.random.default_rng(9)
    d = rng.normal(size=(N, 3)) * DL
    eps = 1e-5
    fd = (_loss_value(a, t, t.pos + eps * d, VN) - _loss_value(a, t, t.pos - eps * d, VN)) / (2 * eps)
    assert rel(np.sum(gx * d), fd) < tol
    ev = 1e-3
    e = np.array([ev, 0.0, 0.0])
    fdv = (_loss_value(a, t, t.pos, VN + e) - _loss_value(a, t, t.pos, VN - e)) / (2 * ev)
    assert rel(gv[0], fdv) < tol


def test_checkpoint_interval_changes_nothing(adj):
    t, a = adj
    g1, v1 = _grads(a, t, every=1)
    for every in (7, 20, 64):
        g, v = _grads(a, t, every=every)
        assert np.max(np.abs(g - g1)) <= 1e-13 * np.max(np.abs(g1))
        assert np.max(np.abs(v - v1)) <= 1e-13 * np.max(np.abs(v1))


def test_interleaved_trajectories_keep_their_own_gradients(adj):
    """Two trajectories of one handle, and a velocity call with another vn,
    before either backward: each gradient equals that of its run alone."""
    import torch
    from openvort_b200.adjoint import centroid_length_loss, trajectory
    t, a = adj
    g1, v1 = _grads(a, t, every=8)
    x0 = torch.tensor(t.pos, dtype=torch.float64, requires_grad=True)
    vn = torch.tensor(VN, dtype=torch.float64, requires_grad=True)
    xf = trajectory(a, x0, vn, 0.0, DT, STEPS, 8)
    x0b = torch.tensor(t.pos * 1.01, dtype=torch.float64, requires_grad=True)
    vnb = torch.tensor(3 * VN, dtype=torch.float64, requires_grad=True)
    xfb = trajectory(a, x0b, vnb, 0.0, DT, STEPS, 4)
    a.velocity(t.pos, -VN)
    centroid_length_loss(xf, t.links[:, 0], t.active, TARGET).backward()
    assert np.max(np.abs(x0.grad.numpy() - g1)) <= 1e-13 * np.max(np.abs(g1))
    assert np.max(np.abs(vn.grad.numpy() - v1)) <= 1e-13 * np.max(np.abs(v1))
    centroid_length_loss(xfb, t.links[:, 0], t.active, TARGET).backward()
    x0c = torch.tensor(t.pos * 1.01, dtype=torch.float64, requires_grad=True)
    vnc = torch.tensor(3 * VN, dtype=torch.float64, requires_grad=True)
    centroid_length_loss(trajectory(a, x0c, vnc, 0.0, DT, STEPS, 4), t.links[:, 0], t.active,
                         TARGET).backward()
    assert np.max(np.abs(x0b.grad.numpy() - x0c.grad.numpy())) <= 1e-13 * np.max(np.abs(x0c.grad.numpy()))
    assert np.max(np.abs(vnb.grad.numpy() - vnc.grad.numpy())) <= 1e-13 * np.max(np.abs(vnc.grad.numpy()))


def test_backward_uses_the_forward_runs_vn(adj):
    """Through the C ABI: a velocity call with another vn between forward
    and backward changes no cotangent (beyond the rounding of the reverse
    passes' accumulation order, as between checkpoint intervals)."""
    t, a = adj
    g = np.random.default_rng(3).normal(size=(N, 3))
    a.forward(t.pos, VN, 0.0, DT, STEPS, 8)
    xb1, vb1 = a.backward(g)
    a.velocity(t.pos, 5 * VN)
    xb2, vb2 = a.backward(g)
    assert np.max(np.abs(xb2 - xb1)) <= 1e-13 * np.max(np.abs(xb1))
    assert np.max(np.abs(vb2 - vb1)) <= 1e-13 * np.max(np.abs(vb1))


def test_adjoint_rejects_unsupported_tangles(ov, monkeypatch):
    monkeypatch.setenv("OV_QUIET", "1")
    lib = ov.load()
    half = G.wall_half_ring()          # pinned ends on a mirror wall
    assert not lib.ov_adjoint_create(half.ptr())
    assert lib.ov_last_error() == ov._lib.OV_ERR_INVALID
    lib.ov_clear_error()
    per = G.rings_to_tangle([G.ring_points((0.05, 0.05, 0.05), (0, 0, 1), 0.01, 64)],
                            (0, 0, 0), (0.1, 0.1, 0.1), "periodic-6")
    assert not lib.ov_adjoint_create(per.ptr())
    assert lib.ov_last_error() == ov._lib.OV_ERR_INVALID
    lib.ov_clear_error()


def test_trajectory_gradient_without_the_colinear_cutoff(ov):
    """The reference's colinearity cut-off (src/tangle.c:505-506) makes the
    velocity discontinuous where a segment's extension passes near a target,
    and with large Kelvin waves finite differences of a trajectory cross
    such jumps.  With the cut-off switched off (ov_set_colinear_cutoff(0),
    FP64 sums and adjoint) the dynamics are smooth, and the gradient of a
    1024-point ring with sigma = 1e-4 cm waves over 50 RK4 steps matches the
    central differences to 1e-6."""
    import torch
    from openvort_b200.adjoint import Adjoint, centroid_length_loss, trajectory
    lib = ov.load()
    assert lib.ov_get_colinear_cutoff() == 1e-8
    n = 1024
    dl = 2 * np.pi * R0 / n
    p = Params(kappa=9.97e-4, core_a=1e-8, use_mf=1, alpha=0.098, alpha_p=0.016, hyperfriction=1,
               max_curv_scale=0.2, hyperalpha=0.5, dl_max=dl / 2,
               vn=Flow("simple", {"external_v": (0.2, 0.0, 0.0)}), vs=Flow("no flow"))
    t = G.rings_to_tangle([G.kelvin_ring(3, n=n, radius=R0, modes=(2, 32), sigma=1e-4)],
                          (-0.05,) * 3, (0.05,) * 3, "open")
    dt, steps, every = 5e-7, 50, 10
    target = np.array([0.0, 0.0, 0.01])
    fwd = t.links[:, 0]
    ov.configure(p, ov.OV_PREC_FP64)
    lib.ov_set_colinear_cutoff(0.0)
    try:
        a = Adjoint(t)
        x0 = torch.tensor(t.pos, dtype=torch.float64, requires_grad=True)
        vn = torch.tensor(VN, dtype=torch.float64, requires_grad=True)
        xf = trajectory(a, x0, vn, 0.0, dt, steps, every)
        centroid_length_loss(xf, fwd, t.active, target).backward()

        def lval(x, v):
            y = a.forward(x, v, 0.0, dt, steps, every)
            return float(centroid_length_loss(torch.from_numpy(y), fwd, t.active, target))
        d = np.random.default_rng(4).normal(size=(n, 3)) * dl
        eps = 1e-5
        fd = (lval(t.pos + eps * d, VN) - lval(t.pos - eps * d, VN)) / (2 * eps)
        assert rel(float(np.sum(x0.grad.numpy() * d)), fd) < 1e-6
        e = np.array([1e-3, 0.0, 0.0])
        fdv = (lval(t.pos, VN + e) - lval(t.pos, VN - e)) / 2e-3
        assert rel(float(vn.grad.numpy()[0]), fdv) < 1e-6
        a.close()
    finally:
        lib.ov_set_colinear_cutoff(1e-8)
        ov.configure(PARAMS, ov.OV_PREC_FP64)
