"""Adjoint of the direct step (csrc/direct_vjp.cu) and of whole trajectories.

* one step: the VJP kernel against plain-PyTorch FP64 autograd of the same
  direct sum (forces with the contact cut, Oseen convection, u = F/(gamma r) + V);
* a trajectory: DirectTrajectory's gradients (initial positions, radii, |E|)
  against plain-PyTorch FP64 autograd of the unrolled steps (<= 1e-9), and
  against FP64 central differences of the library's own FP64 forward (h = 1e-9 m
  for positions): norm-wise relative error over the sampled derivatives
  <= 1e-6, each within 1e-6 of the largest;
* the checkpoint interval does not change the gradients (bit for bit).
Collisions are frozen (no merging), as the adjoint treats them as events."""

from __future__ import annotations

import math

import numpy as np
import pytest

from gpu_util import ETA_OIL, lognormal_state

pytestmark = pytest.mark.gpu

EPS0 = 8.85418781762039e-12
EPS_OIL, ETA_WATER, E_FIELD = 2.85, 0.001, 3e5
FD_TOL = 1e-6


def _torch():
    import torch

    return torch


def torch_velocity(x, r, E, L, periodic=True):
    """u = F / (gamma r) + V of the reference direct step in plain torch FP64."""
    torch = _torch()
    n = x.shape[0]
    m = 12 * math.pi * EPS0 * EPS_OIL * E**2
    eta = 1 / (8 * math.pi * ETA_OIL)
    gamma = 2 * math.pi * ETA_OIL * (2 * ETA_OIL + 3 * ETA_WATER) / (ETA_OIL + ETA_WATER)
    d = x[None, :, :] - x[:, None, :]  # d[i, j] = x_j - x_i
    if periodic:
        d = torch.where(d.abs() > 0.5 * L, d - torch.sign(d) * L, d)
    eye = torch.eye(n, dtype=torch.bool, device=x.device)
    r2 = torch.where(eye, torch.ones_like(d[..., 0]), (d * d).sum(-1))
    rr = torch.sqrt(r2)
    cut = (rr > r[:, None] + r[None, :]) & ~eye
    dx, dy, dz = d[..., 0], d[..., 1], d[..., 2]
    w = torch.where(cut, m * r[:, None] ** 3 * r[None, :] ** 3 / rr**7, torch.zeros_like(rr))
    axy = 4 * dz**2 - dx**2 - dy**2
    F = torch.stack([(w * dx * axy).sum(1), (w * dy * axy).sum(1),
                     (w * dz * (2 * dz**2 - 3 * dx**2 - 3 * dy**2)).sum(1)], 1)
    e = -d
    inv = torch.where(eye, torch.zeros_like(rr), 1 / rr)
    eF = (e * F[None, :, :]).sum(-1)
    V = eta * ((inv[..., None] * F[None, :, :]) + (eF * inv**3)[..., None] * e).sum(1)
    return F / (gamma * r[:, None]) + V


def _state(n, seed):
    torch = _torch()
    pos, r, L = lognormal_state(n, seed=seed)
    return (torch.tensor(pos, dtype=torch.float64, device="cuda"), torch.tensor(r, dtype=torch.float64, device="cuda"),
            L)


def test_step_vjp_matches_torch_autograd():
    torch = _torch()
    from dem import _native as N

    x, r, L = _state(48, seed=21)
    E = torch.tensor(E_FIELD, dtype=torch.float64, device="cuda")
    xg, rg, Eg = x.clone().requires_grad_(), r.clone().requires_grad_(), E.clone().requires_grad_()
    u = torch_velocity(xg, rg, Eg, L)
    lam = torch.randn_like(u, generator=torch.Generator(device="cuda").manual_seed(3))
    gx_ref, gr_ref, gE_ref = torch.autograd.grad((u * lam).sum(), (xg, rg, Eg))

    ctx = N.Context(64)
    m = 12 * math.pi * EPS0 * EPS_OIL * E_FIELD**2
    eta = 1 / (8 * math.pi * ETA_OIL)
    gamma = 2 * math.pi * ETA_OIL * (2 * ETA_OIL + 3 * ETA_WATER) / (ETA_OIL + ETA_WATER)
    pos = x.T.contiguous()
    F = torch.empty_like(pos)
    V = torch.empty_like(pos)
    ctx.direct_forces(48, pos, r, m, L, True, N.PREC_FP64, F)
    ctx.direct_convection(48, pos, r, F, eta, L, True, N.PREC_FP64, V)
    lamT = lam.T.contiguous()
    mu, g, gr = torch.empty_like(pos), torch.empty_like(pos), torch.empty_like(r)
    ctx.direct_vjp(48, pos, r, F, lamT, m, eta, gamma, L, True, mu, g, gr)
    u_dev = (F / (gamma * r) + V).T
    gE = (2 / E_FIELD) * (lam * u_dev).sum()
    torch.testing.assert_close(u_dev, u.detach(), rtol=1e-10, atol=0)
    assert torch.linalg.norm(g.T - gx_ref) / torch.linalg.norm(gx_ref) < 1e-10
    assert torch.linalg.norm(gr - gr_ref) / torch.linalg.norm(gr_ref) < 1e-10
    assert abs(float(gE - gE_ref)) / abs(float(gE_ref)) < 1e-10


def _loss(xT, D, r, L):
    from dem.adjoint import mean_squared_z_displacement, pair_softplus

    torch = _torch()
    w = torch.linspace(-1.0, 1.0, D.numel(), dtype=torch.float64, device=D.device).reshape(D.shape)
    # the displacement term makes every step's VJP matter; the pair term follows the adjoint benchmark
    return 1e8 * (w * D).sum() + 1e16 * mean_squared_z_displacement(D) + pair_softplus(xT, r, L)


def test_trajectory_matches_torch_unrolled():
    torch = _torch()
    from dem.adjoint import DirectTrajectory

    x, r, L = _state(40, seed=22)
    E = torch.tensor(E_FIELD, dtype=torch.float64, device="cuda")
    steps, dt = 6, 1e-3
    sim = DirectTrajectory(L, steps, dt, checkpoint_every=4, precision="fp64", eta_oil=ETA_OIL, eta_water=ETA_WATER,
                           eps_oil=EPS_OIL)
    xg, rg, Eg = x.clone().requires_grad_(), r.clone().requires_grad_(), E.clone().requires_grad_()
    xT, D = sim(xg, rg, Eg)
    gx, gr, gE = torch.autograd.grad(_loss(xT, D, rg, L), (xg, rg, Eg))

    xt, rt, Et = x.clone().requires_grad_(), r.clone().requires_grad_(), E.clone().requires_grad_()
    p, Dt = xt, torch.zeros_like(xt)
    for _ in range(steps):
        u = torch_velocity(p, rt, Et, L)
        p = p + dt * u
        Dt = Dt + dt * u
    torch.testing.assert_close(xT.detach(), p.detach(), rtol=1e-12, atol=1e-18)
    gx2, gr2, gE2 = torch.autograd.grad(_loss(p, Dt, rt, L), (xt, rt, Et))
    assert torch.linalg.norm(gx - gx2) / torch.linalg.norm(gx2) < 1e-9
    assert torch.linalg.norm(gr - gr2) / torch.linalg.norm(gr2) < 1e-9
    assert abs(float(gE - gE2)) / abs(float(gE2)) < 1e-9


def test_trajectory_gradient_matches_central_differences():
    torch = _torch()
    from dem.adjoint import DirectTrajectory

    n, steps, dt = 96, 12, 1e-3
    x, r, L = _state(n, seed=23)
    E = torch.tensor(E_FIELD, dtype=torch.float64, device="cuda")
    sim = DirectTrajectory(L, steps, dt, checkpoint_every=5, precision="fp64", eta_oil=ETA_OIL, eta_water=ETA_WATER,
                           eps_oil=EPS_OIL)

    def loss_of(xx, rr, EE):
        xT, D = sim(xx, rr, EE)
        return _loss(xT, D, rr, L)

    xg, rg, Eg = x.clone().requires_grad_(), r.clone().requires_grad_(), E.clone().requires_grad_()
    gx, gr, gE = torch.autograd.grad(loss_of(xg, rg, Eg), (xg, rg, Eg))
    rng = np.random.default_rng(5)
    coords = [(int(i), int(c)) for i, c in zip(rng.integers(0, n, 16), rng.integers(0, 3, 16))]
    fd, ad = [], []
    with torch.no_grad():
        for i, c in coords:
            h = 1e-9
            xp, xm = x.clone(), x.clone()
            xp[i, c] += h
            xm[i, c] -= h
            fd.append(float(loss_of(xp, r, E) - loss_of(xm, r, E)) / (2 * h))
            ad.append(float(gx[i, c]))
        for i in rng.integers(0, n, 4):
            h = 1e-12
            rp, rm = r.clone(), r.clone()
            rp[i] += h
            rm[i] -= h
            fd.append(float(loss_of(x, rp, E) - loss_of(x, rm, E)) / (2 * h))
            ad.append(float(gr[i]))
        h = 1.0
        fd.append(float(loss_of(x, r, E + h) - loss_of(x, r, E - h)) / (2 * h))
        ad.append(float(gE))
    fd, ad = np.array(fd), np.array(ad)
    # norm-wise over the sampled derivatives, and every one within FD_TOL of the
    # largest (a small derivative carries the central difference's O(h^2) error
    # of the 1 um softplus scale, a few 1e-8 of the largest one)
    assert np.linalg.norm(fd - ad) / np.linalg.norm(fd) <= FD_TOL
    assert np.abs(fd - ad).max() <= FD_TOL * np.abs(fd).max()


def test_checkpoint_interval_does_not_change_gradients():
    torch = _torch()
    from dem.adjoint import DirectTrajectory

    x, r, L = _state(200, seed=24)
    E = torch.tensor(E_FIELD, dtype=torch.float64, device="cuda")
    grads = []
    for C in (1, 3, 7, 10):
        sim = DirectTrajectory(L, 10, 1e-3, checkpoint_every=C, precision="mixed", eta_oil=ETA_OIL,
                               eta_water=ETA_WATER, eps_oil=EPS_OIL)
        xg, rg, Eg = x.clone().requires_grad_(), r.clone().requires_grad_(), E.clone().requires_grad_()
        xT, D = sim(xg, rg, Eg)
        grads.append(torch.autograd.grad(_loss(xT, D, rg, L), (xg, rg, Eg)))
    for g in grads[1:]:
        for a, b in zip(grads[0], g):
            assert torch.equal(a, b)


def test_mixed_forward_gradient_close_to_fp64():
    torch = _torch()
    from dem.adjoint import DirectTrajectory

    x, r, L = _state(1000, seed=25)
    E = torch.tensor(E_FIELD, dtype=torch.float64, device="cuda")
    out = {}
    for prec in ("fp64", "mixed"):
        sim = DirectTrajectory(L, 8, 1e-3, checkpoint_every=4, precision=prec, eta_oil=ETA_OIL, eta_water=ETA_WATER,
                               eps_oil=EPS_OIL)
        xg, rg, Eg = x.clone().requires_grad_(), r.clone().requires_grad_(), E.clone().requires_grad_()
        xT, D = sim(xg, rg, Eg)
        out[prec] = torch.autograd.grad(_loss(xT, D, rg, L), (xg, rg, Eg))
    for a, b in zip(out["mixed"], out["fp64"]):
        assert float(torch.linalg.norm(a - b) / torch.linalg.norm(b)) < 1e-4


def test_open_box_gradient_matches_central_differences_n2048():
    # In a periodic box the minimum image of a pair switches when a separation
    # crosses L/2, a jump that central differences see once N is large; the open
    # box keeps the forward map smooth, so the same bound holds at larger N.
    torch = _torch()
    from dem.adjoint import DirectTrajectory, mean_squared_z_displacement, pair_softplus

    n, steps = 2048, 30
    x, r, L = _state(n, seed=26)
    E = torch.tensor(E_FIELD, dtype=torch.float64, device="cuda")
    sim = DirectTrajectory(L, steps, 1e-4, checkpoint_every=7, precision="fp64", eta_oil=ETA_OIL,
                           eta_water=ETA_WATER, eps_oil=EPS_OIL, boundary_mode="open")

    def loss_of(xx):
        xT, D = sim(xx, r, E)
        return mean_squared_z_displacement(D) + pair_softplus(xT, r, L, periodic=False)

    xg = x.clone().requires_grad_()
    (gx,) = torch.autograd.grad(loss_of(xg), (xg,))
    rng = np.random.default_rng(9)
    fd, ad = [], []
    with torch.no_grad():
        for i, c in zip(rng.integers(0, n, 12), rng.integers(0, 3, 12)):
            h = 1e-9
            xp, xm = x.clone(), x.clone()
            xp[i, c] += h
            xm[i, c] -= h
            fd.append(float(loss_of(xp) - loss_of(xm)) / (2 * h))
            ad.append(float(gx[i, c]))
    fd, ad = np.array(fd), np.array(ad)
    assert np.linalg.norm(fd - ad) / np.linalg.norm(fd) <= FD_TOL
    assert np.abs(fd - ad).max() <= FD_TOL * np.abs(fd).max()
