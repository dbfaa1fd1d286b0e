"""Differentiable direct DEM trajectories: adjoint through the Euler steps.

The direct step of the reference solver (euler_droplet_solver.py:121-131)
moves every droplet with u = F / (gamma r) + V, F the dipole forces and V their
Oseen convection.  ``DirectTrajectory`` runs K such steps on the GPU and is a
``torch.autograd.Function``: its backward pass walks the steps in reverse with
the hand-written VJP kernel of the library (csrc/direct_vjp.cu, FP64), giving
gradients with respect to the initial positions, the radii and the field |E|.

* Collisions are frozen (no detection, no merging): they are events, not
  differentiable operations.
* Positions are integrated without the periodic wrap (``x %= L`` changes no
  distance: the force and Oseen passes use the minimum image), so the output
  x_T and the accumulated displacement D = sum_t dt u_t are smooth functions of
  the inputs.
* Memory: every ``checkpoint_every`` steps the state is kept; the backward pass
  recomputes each segment forward (same kernels, same results) and then steps
  back through it.
* ``precision`` selects the forward force/convection passes ("fp64": the
  reference drop-in, "mixed": FP32 pair terms); the VJP is FP64 either way.
"""

from __future__ import annotations

import numpy as np

from .. import _native as N
from ..force_calculator.direct_droplet_force_calculator import EPS0


class DirectTrajectory:
    def __init__(self, L, steps, dt, *, checkpoint_every=20, precision="mixed", eps_oil=2.85, eta_oil=0.065,
                 eta_water=0.001, boundary_mode="periodic", device=None):
        if precision not in N.PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(N.PRECISIONS)}")
        if steps < 0 or checkpoint_every < 1:
            raise ValueError("steps >= 0 and checkpoint_every >= 1 are required")
        self.L, self.steps, self.dt = float(L), int(steps), float(dt)
        self.checkpoint_every = int(checkpoint_every)
        self.precision = N.PRECISIONS[precision]
        self.eps_oil, self.eta_oil, self.eta_water = eps_oil, eta_oil, eta_water
        self.eta_const = 1 / (8 * np.pi * eta_oil)
        self.stokes_factor = 2 * np.pi * eta_oil * (2 * eta_oil + 3 * eta_water) / (eta_oil + eta_water)
        self.periodic = boundary_mode == "periodic"
        self.device = device
        self._ctx = None

    def m_const(self, E):
        return 12 * np.pi * EPS0 * self.eps_oil * float(E) ** 2

    def context(self, n):
        if self._ctx is None:
            self._ctx = N.Context(max(n, 1), self.device)
        elif self._ctx.capacity < n:
            self._ctx.reserve(n)
        return self._ctx

    def __call__(self, x0, r, E):
        """x0 (N, 3), r (N,), E (scalar tensor) CUDA float64 tensors -> (x_T, D), both (N, 3)."""
        return _fn().apply(x0, r, E, self)

    # -- device helpers (SoA (3, n) tensors) -------------------------------------
    def velocity_parts(self, ctx, n, pos, r, m, F, V):
        ctx.direct_forces(n, pos, r, m, self.L, self.periodic, self.precision, F)
        ctx.direct_convection(n, pos, r, F, self.eta_const, self.L, self.periodic, self.precision, V)

    def advance(self, ctx, n, pos, r, F, V, D):
        """pos += dt u and D += dt u (no wrap), u = F / (gamma r) + V."""
        ctx.euler_update(n, pos, r, F, V, self.stokes_factor, self.dt, self.L, False, pos)
        ctx.euler_update(n, D, r, F, V, self.stokes_factor, self.dt, self.L, False, D)


def _make_fn():
    import torch

    class TrajectoryFn(torch.autograd.Function):
        @staticmethod
        def forward(fctx, x0, r, E, sim):
            n = x0.shape[0]
            ctx = sim.context(n)
            dev = ctx.device
            pos = x0.detach().to(device=dev, dtype=torch.float64).T.contiguous()
            rr = r.detach().to(device=dev, dtype=torch.float64).contiguous()
            Ef = float(E)
            m = sim.m_const(Ef)
            F = torch.empty_like(pos)
            V = torch.empty_like(pos)
            D = torch.zeros_like(pos)
            checkpoints = []
            for t in range(sim.steps):
                if t % sim.checkpoint_every == 0:
                    checkpoints.append(pos.clone())
                sim.velocity_parts(ctx, n, pos, rr, m, F, V)
                sim.advance(ctx, n, pos, rr, F, V, D)
            fctx.sim = sim
            fctx.E = Ef
            fctx.checkpoints = checkpoints
            fctx.save_for_backward(rr)
            return pos.T.contiguous(), D.T.contiguous()

        @staticmethod
        def backward(fctx, g_xT, g_D):
            sim = fctx.sim
            (rr,) = fctx.saved_tensors
            n = rr.shape[0]
            ctx = sim.context(n)
            Ef = fctx.E
            m = sim.m_const(Ef)
            lam_x = (g_xT.T.contiguous().clone() if g_xT is not None
                     else torch.zeros((3, n), dtype=torch.float64, device=rr.device))
            lam_d = (g_D.T.contiguous() if g_D is not None
                     else torch.zeros((3, n), dtype=torch.float64, device=rr.device))
            gr = torch.zeros(n, dtype=torch.float64, device=rr.device)
            gE = torch.zeros((), dtype=torch.float64, device=rr.device)
            mu = torch.empty((3, n), dtype=torch.float64, device=rr.device)
            g = torch.empty((3, n), dtype=torch.float64, device=rr.device)
            grr = torch.empty(n, dtype=torch.float64, device=rr.device)
            C = sim.checkpoint_every
            for seg in range(len(fctx.checkpoints) - 1, -1, -1):
                s0 = seg * C
                s1 = min(sim.steps, s0 + C)
                # recompute the segment: states, forces and convection of every step
                pos = fctx.checkpoints[seg].clone()
                states, Fs, Vs = [], [], []
                D = torch.zeros_like(pos)
                for _ in range(s0, s1):
                    F = torch.empty_like(pos)
                    V = torch.empty_like(pos)
                    sim.velocity_parts(ctx, n, pos, rr, m, F, V)
                    states.append(pos.clone())
                    Fs.append(F)
                    Vs.append(V)
                    sim.advance(ctx, n, pos, rr, F, V, D)
                for k in range(len(states) - 1, -1, -1):
                    lam_u = (lam_x + lam_d) * sim.dt  # cotangent on u_t
                    ctx.direct_vjp(n, states[k], rr, Fs[k], lam_u, m, sim.eta_const, sim.stokes_factor, sim.L,
                                   sim.periodic, mu, g, grr)
                    u = Fs[k] / (sim.stokes_factor * rr) + Vs[k]
                    gE += (2.0 / Ef) * (lam_u * u).sum()
                    lam_x += g
                    gr += grr
            return lam_x.T.contiguous(), gr, gE, None

    return TrajectoryFn


_fn_cache = {}


def _fn():
    if "fn" not in _fn_cache:
        _fn_cache["fn"] = _make_fn()
    return _fn_cache["fn"]


# ---------------------------------------------------------------------------
# losses of the adjoint benchmark (plain torch on the device)
# ---------------------------------------------------------------------------
def mean_squared_z_displacement(D):
    """mean_i D_z,i^2 of the accumulated (unwrapped) displacement."""
    return (D[:, 2] ** 2).mean()


def pair_softplus(x, r, L, periodic=True, factor=2.5, scale=1e-6, chunk=512):
    """sum over pairs i < j of softplus((factor (r_i + r_j) - |x_i - x_j|) / scale),
    minimum-image distances in a periodic box."""
    import torch

    n = x.shape[0]
    total = x.new_zeros(())
    idx = torch.arange(n, device=x.device)
    for i0 in range(0, n, chunk):
        i1 = min(n, i0 + chunk)
        d = x[None, :, :] - x[i0:i1, None, :]
        if periodic:
            d = torch.where(d.abs() > 0.5 * L, d - torch.sign(d) * L, d)
        upper = idx[None, :] > idx[i0:i1, None]
        dist = torch.sqrt(torch.where(upper, (d * d).sum(-1), torch.ones_like(d[..., 0])))
        u = (factor * (r[i0:i1, None] + r[None, :]) - dist) / scale
        total = total + torch.where(upper, torch.nn.functional.softplus(u), torch.zeros_like(u)).sum()
    return total
