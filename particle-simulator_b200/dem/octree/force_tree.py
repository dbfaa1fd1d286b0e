"""Barnes-Hut force calculator on the B200.

Drop-in for dem/octree/force_tree.py:18-244 of ddkx21/particle-simulator:
same constructor, attributes and methods, with the flat octree of
``flat_tree.FlatOctree`` (CUDA, FP64, bit-identical to the reference's
expressions).
"""

from __future__ import annotations

import numpy as np

from ..force_calculator.force_calculator_base import ForceCalculator
from .flat_tree import FlatOctree

EPS0 = 8.85418781762039e-12  # force_tree.py:44


class TreeDropletForceCalculator(ForceCalculator):
    def __init__(self, num_particles: int = 10000, theta: float = 0.5, mpl: int = 1, eps_oil: float = 2.85,
                 eta_oil: float = 0.065, eta_water: float = 0.001, E: float = 3e5, L: float = 1.0,
                 periodic: bool = False, correction_grid_resolution: int = 0, *, device=None):
        self.eps0 = EPS0
        self.eps_oil = eps_oil
        self.eta_oil = eta_oil
        self.eta_water = eta_water
        self.E = E
        self.L = L
        self.periodic = periodic
        self.boundary_mode = "periodic" if periodic else "open"
        self.m_const = 12.0 * np.pi * self.eps0 * eps_oil * E**2  # :54
        self.eta_const = 1.0 / (8.0 * np.pi * eta_oil)  # :57
        self.num_particles = num_particles
        self.theta = theta
        self.mpl = mpl
        self.correction_grid_resolution = correction_grid_resolution
        self._device = device
        self.octree = FlatOctree(theta=theta, mpl=mpl, num_particles=num_particles,
                                 correction_grid_resolution=correction_grid_resolution, device=device)
        self._ctx = self.octree._ctx
        self._tree_is_stale = True
        self._forces_in_fields = False
        self._correction = None
        self._correction_L_sim = None

    def update_params(self, theta: float, mpl: int) -> None:
        self.theta = theta
        self.mpl = mpl
        self.octree.update_params(theta, mpl)
        self._tree_is_stale = True

    def _ensure_octree_capacity(self, n: int) -> None:
        """force_tree.py:92-106."""
        if n > self.num_particles:
            self.octree = FlatOctree(theta=self.theta, mpl=self.mpl, num_particles=n,
                                     correction_grid_resolution=self.correction_grid_resolution,
                                     device=self._device)
            self._ctx = self.octree._ctx
            self.num_particles = n
            if self._correction is not None:  # :103-106
                self.octree.load_periodic_correction(self._correction, self._correction_L_sim, eta_sim=self.eta_oil)

    def load_periodic_correction(self, correction, L_sim: float):
        self._correction = correction
        self._correction_L_sim = L_sim
        self.octree.load_periodic_correction(correction, L_sim, eta_sim=self.eta_oil)

    def _box(self, L, periodic):
        return (L if L is not None else self.L), (periodic if periodic is not None else self.periodic)

    def calculate(self, positions, radii, *, L: float | None = None, periodic: bool | None = None):
        """force_tree.py:114-141."""
        use_L, use_p = self._box(L, periodic)
        self._ensure_octree_capacity(len(radii))
        self.octree.build(positions, radii, use_L, use_p)
        self._tree_is_stale = False
        self._forces_in_fields = True
        return self.octree.compute_forces(self.m_const)

    def calculate_convection(self, positions, radii, forces, *, L: float | None = None,
                             periodic: bool | None = None):
        """force_tree.py:143-182."""
        use_L, use_p = self._box(L, periodic)
        if self._tree_is_stale:
            self._ensure_octree_capacity(len(radii))
            self.octree.build(positions, radii, use_L, use_p)
            self._tree_is_stale = False
        if self._forces_in_fields:
            v = self.octree.compute_stokeslet_from_fields(forces, self.eta_const)
        else:
            v = self.octree.compute_stokeslet(forces, self.eta_const)
        self._tree_is_stale = True
        self._forces_in_fields = False
        return v

    def calculate_forces_and_convection(self, positions, radii, *, L: float | None = None,
                                        periodic: bool | None = None) -> tuple:
        """force_tree.py:184-213."""
        use_L, use_p = self._box(L, periodic)
        self._ensure_octree_capacity(len(radii))
        self.octree.build(positions, radii, use_L, use_p)
        self._tree_is_stale = True
        return self.octree.compute_forces_and_stokeslet(self.m_const, self.eta_const)

    def calculate_forces_and_total_velocity(self, positions, radii, stokes_factor: float, *,
                                            L: float | None = None, periodic: bool | None = None) -> tuple:
        """force_tree.py:215-244."""
        use_L, use_p = self._box(L, periodic)
        self._ensure_octree_capacity(len(radii))
        self.octree.build(positions, radii, use_L, use_p)
        self._tree_is_stale = True
        return self.octree.compute_forces_and_total_velocity(self.m_const, self.eta_const, stokes_factor)

    # -- device-resident interface used by the solver ------------------------
    def forces_and_total_velocity_soa(self, n, pos_soa, r, stokes_factor):
        self._ensure_octree_capacity(n)
        self.octree.build_soa(n, pos_soa, r, self.L, self.periodic)
        self._tree_is_stale = True
        _, V = self.octree.total_velocity_soa(self.m_const, self.eta_const, stokes_factor)
        return V
