"""Barnes-Hut calculator on a Morton-key octree (the fast form of dem/octree).

Same constructor and methods as ``TreeDropletForceCalculator``
(dem/octree/force_tree.py:18-244 of the reference) -- ``calculate``,
``calculate_convection``, ``calculate_forces_and_convection``,
``calculate_forces_and_total_velocity``, ``update_params`` -- on the octree of
csrc/bh.cu: 30-bit Morton keys, on-device radix sort, level-by-level build from
key prefixes, warp-cooperative FP32 walks with FP64 separations.  ``mpl`` is
the leaf size (droplets per leaf; default 16).  ``window_level`` (periodic
boxes): cells larger than L / 2^window_level are opened unless they lie wholly
inside the target's minimum-image window (0, the default: the reference's
rule).  ``load_periodic_correction`` adds the periodic-image correction to
the velocity walk (FP32 terms at leaf pairs and accepted nodes).  Results
approximate the direct sums; the reference-parity FP64 tree is
``TreeDropletForceCalculator``.
"""

from __future__ import annotations

import numpy as np

from .. import _native as N
from .._io import Stager
from ..force_calculator.force_calculator_base import ForceCalculator
from ..periodic_correction.comsol_lattice_correction import correction_fields, to_device

EPS0 = 8.85418781762039e-12  # force_tree.py:44


class MortonTreeForceCalculator(ForceCalculator):
    def __init__(self, num_particles: int = 10000, theta: float = 0.5, mpl: int = 16, eps_oil: float = 2.85,
                 eta_oil: float = 0.065, eta_water: float = 0.001, E: float = 3e5, L: float = 1.0,
                 periodic: bool = False, correction_grid_resolution: int = 0, *, window_level: int = 0,
                 device=None):
        self.eps0 = EPS0
        self.eps_oil, self.eta_oil, self.eta_water, self.E = eps_oil, eta_oil, eta_water, E
        self.L = L
        self.periodic = periodic
        self.boundary_mode = "periodic" if periodic else "open"
        self.m_const = 12.0 * np.pi * self.eps0 * eps_oil * E**2
        self.eta_const = 1.0 / (8.0 * np.pi * eta_oil)
        self.num_particles = num_particles
        self.theta = theta
        self.mpl = mpl
        self.correction_grid_resolution = correction_grid_resolution
        self._ctx = N.Context(max(num_particles, 1), device)
        self._io = Stager(self._ctx)
        self.window_level = window_level
        self.tree = N.MortonTree(self._ctx, max(num_particles, 1))
        self.tree.set_window(window_level)
        self._corr = None
        self.__dict__.update(correction_fields(None))

    def load_periodic_correction(self, correction, L_sim: float):
        """force_tree.py:108-112 (eta ratio from this calculator's eta_oil)."""
        if self.correction_grid_resolution == 0:
            raise RuntimeError("correction_grid_resolution=0: correction grids were not allocated.")
        self._corr, scalars = to_device(self._ctx, correction, L_sim, self.eta_oil,
                                        max(self.correction_grid_resolution, 2))
        self.tree.set_correction(self._corr)
        self.__dict__.update(correction_fields(scalars))

    def update_params(self, theta: float, mpl: int) -> None:
        self.theta = theta
        self.mpl = mpl

    def _ensure(self, n):
        if n > self.tree.capacity:
            self._ctx.reserve(n)
            self.tree = N.MortonTree(self._ctx, n)
            self.tree.set_window(self.window_level)
            self.tree.set_correction(self._corr)
            self.num_particles = n

    def _box(self, L, periodic):
        return (L if L is not None else self.L), (periodic if periodic is not None else self.periodic)

    def _build(self, positions, radii, L, periodic):
        st, dev = self._io.positions(positions, radii)
        self._ensure(st.n)
        self.tree.build(st.n, st.pos, st.r, L, periodic, self.mpl)
        return st, dev

    def _out(self, soas, n, dev):
        if dev:
            return [self._io.to_aos_tensor(a, n) for a in soas]
        return self._io.download(soas, n)

    def _forces(self, st):
        F = self._io.buf.dev("F", (3, st.n))
        self.tree.forces(self.m_const, self.theta, F)
        return F

    def calculate(self, positions, radii, *, L: float | None = None, periodic: bool | None = None):
        use_L, use_p = self._box(L, periodic)
        st, dev = self._build(positions, radii, use_L, use_p)
        return self._out([self._forces(st)], st.n, dev)[0]

    def calculate_convection(self, positions, radii, forces, *, L: float | None = None,
                             periodic: bool | None = None):
        use_L, use_p = self._box(L, periodic)
        st, dev = self._build(positions, radii, use_L, use_p)
        F = self._io.vectors(forces, st.n, "Fin")
        V = self._io.buf.dev("V", (3, st.n))
        self.tree.velocity(F, self.eta_const, self.theta, 0.0, V)
        return self._out([V], st.n, dev)[0]

    def calculate_forces_and_convection(self, positions, radii, *, L: float | None = None,
                                        periodic: bool | None = None) -> tuple:
        use_L, use_p = self._box(L, periodic)
        st, dev = self._build(positions, radii, use_L, use_p)
        F = self._forces(st)
        V = self._io.buf.dev("V", (3, st.n))
        self.tree.velocity(None, self.eta_const, self.theta, 0.0, V)
        return tuple(self._out([F, V], st.n, dev))

    def calculate_forces_and_total_velocity(self, positions, radii, stokes_factor: float, *,
                                            L: float | None = None, periodic: bool | None = None) -> tuple:
        use_L, use_p = self._box(L, periodic)
        st, dev = self._build(positions, radii, use_L, use_p)
        F = self._forces(st)
        V = self._io.buf.dev("V", (3, st.n))
        self.tree.velocity(None, self.eta_const, self.theta, stokes_factor, V)
        return tuple(self._out([F, V], st.n, dev))

    # -- device-resident interface (SoA (3, n) tensors) --------------------------
    def forces_and_total_velocity_soa(self, n, pos_soa, r, stokes_factor):
        self._ensure(n)
        self.tree.build(n, pos_soa, r, self.L, self.periodic, self.mpl)
        F = self._io.buf.dev("F", (3, n))
        self.tree.forces(self.m_const, self.theta, F)
        V = self._io.buf.dev("V", (3, n))
        self.tree.velocity(None, self.eta_const, self.theta, stokes_factor, V)
        return V

    def stats(self):
        return self.tree.stats()
