"""Ensembles of independent droplet boxes stepped together on one GPU.

The reference's ``main_multi.py:52-77`` runs one simulation per initial state
and time step, one after another: a ``DirectDropletForceCalculator`` and an
``EulerDropletSolver`` without a collision detector for each.  An ensemble
holds many such boxes (uneven droplet counts, one side ``L`` per box) and
advances all of them with one set of launches per pass:

* the mixed-precision direct force and Oseen passes walk the block pairs of
  every box in one launch of the symmetric pair kernel (a persistent grid when
  the autotuner prefers one);
* one Euler launch moves every droplet with its own box's side
  (``euler_droplet_solver.py:121-131`` per box);
* a step can be captured once as a CUDA graph and replayed;
* ``autotune`` times the candidate tilings (block size 256 / 512 droplets,
  one CTA per block pair or a persistent grid) on the ensemble itself.

Per box the forces and velocities are bit-identical to
``DirectDropletForceCalculator(precision="mixed")`` with the symmetric
schedule and the same block size.
"""

from __future__ import annotations

import numpy as np

from .. import _native as N
from ..force_calculator.direct_droplet_force_calculator import EPS0


def stokes_factor(eta_oil, eta_water):
    """gamma of euler_droplet_solver.py:39-41."""
    return 2 * np.pi * eta_oil * (2 * eta_oil + 3 * eta_water) / (eta_oil + eta_water)


class DropletEnsemble:
    def __init__(self, states, L, eps_oil=2.85, eta_oil=0.065, eta_water=0.001, rho_water=1000, rho_oil=910,
                 E=3e5, boundary_mode="periodic", *, device=None):
        """states: sequence of (positions (n_b, 3), radii (n_b,)) per box;
        L: one side for all boxes or one per box."""
        states = list(states)
        if not states:
            raise ValueError("an ensemble needs at least one box")
        self.eps_oil, self.eta_oil, self.eta_water, self.E = eps_oil, eta_oil, eta_water, E
        self.rho_water, self.rho_oil = rho_water, rho_oil
        self.m_const = 12 * np.pi * EPS0 * eps_oil * E**2
        self.eta_const = 1 / (8 * np.pi * eta_oil)
        self.stokes_factor = stokes_factor(eta_oil, eta_water)
        if boundary_mode not in ("periodic", "open"):
            raise ValueError("boundary_mode must be 'periodic' or 'open'")
        self.boundary_mode = boundary_mode
        counts = [len(np.asarray(r).reshape(-1)) for _, r in states]
        self.offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        self.nbox = len(states)
        Ls = np.broadcast_to(np.asarray(L, dtype=np.float64), (self.nbox,)).copy()
        self.L = Ls
        pos = np.concatenate([np.asarray(p, dtype=np.float64).reshape(-1, 3) for p, _ in states]) if self.n else \
            np.zeros((0, 3))
        rad = np.concatenate([np.asarray(r, dtype=np.float64).reshape(-1) for _, r in states]) if self.n else \
            np.zeros(0)
        self.ctx = N.Context(max(self.n, 1), device)
        torch = self.ctx.torch
        self.torch = torch
        dev = self.ctx.device
        self.pos = torch.as_tensor(np.ascontiguousarray(pos.T), device=dev).contiguous()  # (3, n) SoA
        self.r = torch.as_tensor(rad, device=dev).contiguous()
        self.F = torch.zeros((3, self.n), dtype=torch.float64, device=dev)
        self.V = torch.zeros((3, self.n), dtype=torch.float64, device=dev)
        self.batch = N.Batch(self.ctx, self.offsets, Ls, boundary_mode == "periodic")
        self._graph_dt = None

    # -- sizes -----------------------------------------------------------------
    @property
    def n(self) -> int:
        return int(self.offsets[-1])

    def box_slice(self, b):
        return slice(int(self.offsets[b]), int(self.offsets[b + 1]))

    # -- tuning ------------------------------------------------------------------
    def set_tuning(self, i_per_thread=4, ctas=0):
        self.batch.set_tuning(i_per_thread, ctas)
        self._graph_dt = None  # a captured graph holds the old launch shapes

    def get_tuning(self):
        return self.batch.get_tuning()

    def autotune(self, reps=3):
        """Times every candidate tiling on the current state, keeps the fastest;
        returns it with its time per force + convection pair of passes (ms)."""
        ms = self.batch.autotune(self.pos, self.r, self.m_const, self.eta_const, self.F, self.V, reps)
        self._graph_dt = None
        return dict(self.get_tuning(), ms=ms)

    # -- physics -----------------------------------------------------------------
    def compute(self):
        """Forces and convection velocities of the current state (device, SoA)."""
        self.batch.forces(self.pos, self.r, self.m_const, self.F)
        self.batch.convection(self.pos, self.r, self.F, self.eta_const, self.V)
        return self.F, self.V

    def forces_and_convection(self):
        """Per box (forces (n_b, 3), velocities (n_b, 3)) as numpy arrays."""
        F, V = self.compute()
        Fh, Vh = F.T.cpu().numpy(), V.T.cpu().numpy()
        return [(Fh[self.box_slice(b)], Vh[self.box_slice(b)]) for b in range(self.nbox)]

    def step(self, dt, steps=1, graph=False):
        """Advances every box by `steps` Euler steps of size dt (in place).
        graph=True records one step as a CUDA graph (once per dt) and replays it."""
        if not graph:
            for _ in range(int(steps)):
                self.batch.step(self.pos, self.r, self.m_const, self.eta_const, self.stokes_factor, dt, self.F,
                                self.V)
            return
        if self._graph_dt != dt:
            self.batch.capture(self.pos, self.r, self.m_const, self.eta_const, self.stokes_factor, dt, self.F,
                               self.V)
            self._graph_dt = dt
        self.batch.replay(int(steps))

    def step_sequential(self, dt, steps=1):
        """The same steps as plain per-box launches, one box after another (what
        main_multi.py does): one force, convection and Euler call per box."""
        ctx = self.ctx
        for _ in range(int(steps)):
            for b in range(self.nbox):
                s = self.box_slice(b)
                nb = s.stop - s.start
                if nb == 0:
                    continue
                pos = [self.pos[c, s] for c in range(3)]
                F = [self.F[c, s] for c in range(3)]
                V = [self.V[c, s] for c in range(3)]
                per = self.boundary_mode == "periodic"
                ctx.direct_forces(nb, pos, self.r[s], self.m_const, self.L[b], per, N.PREC_MIXED, F)
                ctx.direct_convection(nb, pos, self.r[s], F, self.eta_const, self.L[b], per, N.PREC_MIXED, V)
                ctx.euler_update(nb, pos, self.r[s], F, V, self.stokes_factor, dt, self.L[b], per, pos)

    def positions(self):
        """Per box positions (n_b, 3) as numpy arrays."""
        P = self.pos.T.cpu().numpy()
        return [P[self.box_slice(b)].copy() for b in range(self.nbox)]

    def radii(self):
        R = self.r.cpu().numpy()
        return [R[self.box_slice(b)].copy() for b in range(self.nbox)]
