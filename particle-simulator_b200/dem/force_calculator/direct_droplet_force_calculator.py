"""Direct O(N^2) dipole force and Oseen convection on the B200.

Drop-in for dem/force_calculator/direct_droplet_force_calculator.py:8-527 of
ddkx21/particle-simulator: same constructor, attributes and methods.  The
O(N^2) passes run in the CUDA kernels of libdem_b200 (csrc/direct_fp64.cu,
csrc/direct_mixed.cu):

* ``precision="fp64"`` (default) is the reference drop-in: it evaluates every
  pair with the reference's expressions and summation order and is
  bit-identical to the reference's kernels run in IEEE binary64;
* ``precision="mixed"`` evaluates pair terms in FP32 with compensated sums and
  recomputes near-contact pairs in FP64 (relative force error ~1e-7 norm-wise).

With ``load_periodic_correction`` the convection adds the periodic-image
correction of every pair and the self term (:413-464), in FP64 bit-identical
to the reference's order or, with ``precision="mixed"``, as an FP32 pass
(csrc/corr.cu).

Inputs may be numpy arrays (results come back as numpy, as in the reference)
or CUDA torch tensors (results stay on the device as torch tensors).
"""

from __future__ import annotations

import numpy as np

from .. import _native as N
from .._io import Stager
from ..periodic_correction.comsol_lattice_correction import correction_fields, to_device
from .force_calculator_base import ForceCalculator

EPS0 = 8.85418781762039e-12  # reference value, direct_droplet_force_calculator.py:23


class DirectDropletForceCalculator(ForceCalculator):
    def __init__(
        self,
        num_particles=10000,
        eps_oil=2.85,
        eta_oil=0.065,
        eta_water=0.001,
        rho_water=1000,
        rho_oil=910,
        E=3e5,
        L=1.0,
        boundary_mode="periodic",
        correction_grid_resolution=0,
        *,
        precision: str = "fp64",
        device=None,
    ):
        self.eps0 = EPS0
        self.eps_oil = eps_oil
        self.eta_oil = eta_oil
        self.eta_water = eta_water
        self.rho_water = rho_water
        self.rho_oil = rho_oil
        self.E = E
        self.m_const = 12 * np.pi * self.eps0 * eps_oil * E**2  # :30
        self.eta_const = 1 / (8 * np.pi * self.eta_oil)  # :31
        self.L = L
        self.boundary_mode = boundary_mode
        self.num_particles = num_particles
        self.correction_grid_resolution = correction_grid_resolution
        if precision not in N.PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(N.PRECISIONS)}")
        self.precision = precision
        self._ctx = N.Context(max(int(num_particles), 1), device)
        self._io = Stager(self._ctx)
        self._corr = None  # device grid of the periodic-image correction
        self.__dict__.update(correction_fields(None))

    # -- reference API ------------------------------------------------------
    def load_periodic_correction(self, correction, L_sim: float):
        """dem/force_calculator/direct_droplet_force_calculator.py:74-120: uploads the
        grid; from then on every convection call adds the correction."""
        if self.correction_grid_resolution == 0:
            raise RuntimeError(
                "correction_grid_resolution=0: correction grids were not allocated; "
                "re-create DirectDropletForceCalculator with correction_grid_resolution > 0."
            )
        self._corr, scalars = to_device(self._ctx, correction, L_sim, self.eta_oil,
                                        max(self.correction_grid_resolution, 2))
        self.__dict__.update(correction_fields(scalars))

    @property
    def periodic(self) -> bool:
        return self.boundary_mode == "periodic"

    def _reserve(self, n):
        if n > self._ctx.capacity:
            self._ctx.reserve(n)

    def _forces_dev(self, st):
        F = self._io.buf.dev("forces", (3, st.n))
        self._ctx.direct_forces(st.n, st.pos, st.r, self.m_const, self.L, self.periodic,
                                N.PRECISIONS[self.precision], F)
        return F

    def _convection_dev(self, st, F):
        V = self._io.buf.dev("velocities", (3, st.n))
        if self._corr is not None:
            self._ctx.direct_convection_corr(self._corr, st.n, st.pos, st.r, F, self.eta_const, self.L,
                                             self.periodic, N.PRECISIONS[self.precision], V)
        else:
            self._ctx.direct_convection(st.n, st.pos, st.r, F, self.eta_const, self.L, self.periodic,
                                        N.PRECISIONS[self.precision], V)
        return V

    def _both_dev(self, st):
        """Forces and the convection of those forces on one state (one library call
        without the correction: the convection pass reuses the force pass's droplet order)."""
        if self._corr is not None:
            F = self._forces_dev(st)
            return F, self._convection_dev(st, F)
        F = self._io.buf.dev("forces", (3, st.n))
        V = self._io.buf.dev("velocities", (3, st.n))
        self._ctx.direct_forces_and_convection(st.n, st.pos, st.r, self.m_const, self.eta_const, self.L,
                                               self.periodic, N.PRECISIONS[self.precision], F, V)
        return F, V

    def calculate(self, positions, radii):
        """Forces (N, 3): direct_droplet_force_calculator.py:260-305."""
        self.num_particles = len(radii)
        self._reserve(self.num_particles)
        st, on_dev = self._io.positions(positions, radii)
        F = self._forces_dev(st)
        if on_dev:
            return self._io.to_aos_tensor(F, st.n)
        return self._io.download([F], st.n)[0]

    def calculate_convection(self, positions, radii, forces):
        """Convection velocities (N, 3): direct_droplet_force_calculator.py:307-352."""
        self.num_particles = len(radii)
        self._reserve(self.num_particles)
        st, on_dev = self._io.positions(positions, radii)
        F = self._io.vectors(forces, st.n, "forces_in")
        V = self._convection_dev(st, F)
        if on_dev:
            return self._io.to_aos_tensor(V, st.n)
        return self._io.download([V], st.n)[0]

    def calculate_forces_and_convection(self, positions, radii) -> tuple:
        """(forces, velocities): direct_droplet_force_calculator.py:470-527."""
        self.num_particles = len(radii)
        self._reserve(self.num_particles)
        st, on_dev = self._io.positions(positions, radii)
        F, V = self._both_dev(st)
        if on_dev:
            return self._io.to_aos_tensor(F, st.n), self._io.to_aos_tensor(V, st.n)
        f, v = self._io.download([F, V], st.n)
        return f, v

    # -- device-resident interface used by the solver ------------------------
    def forces_and_convection_soa(self, n, pos_soa, r):
        """SoA device tensors in, SoA device tensors out (no host traffic)."""
        self._reserve(n)

        class _S:
            pass

        st = _S()
        st.n, st.pos, st.r = n, pos_soa, r
        return self._both_dev(st)

    def set_tuning(self, **kw):
        """Tune the mixed-precision kernels (see dem_direct_set_tuning)."""
        self._ctx.set_tuning(**kw)

    def get_tuning(self):
        return self._ctx.get_tuning()
