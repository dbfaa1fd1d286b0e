"""Uniform droplet generator with overlap rejection on the B200.

Drop-in for dem/particle_generator/uniform_droplet_generator.py:11-164 of
ddkx21/particle-simulator: same constructor and ``generate()``.  The rejection
loop runs on the device (csrc/gen.cu): every round re-draws the droplets just
drawn that overlap any droplet, found with the spatial hash instead of the
reference's all-pairs loop, until no overlap is left (ValueError after 1,000
rounds, as in the reference).  The reference's generator is unseeded
(``np.random`` + ``ti.random()``); here ``seed`` fixes the state (``None``
draws one from the operating system).  ``periodic=True`` tests overlaps with
the minimum image in the cube [coord_range)^3 (the reference uses the plain
distance).
"""

from __future__ import annotations

import numpy as np

from .. import _native as N
from ..particle_state import DropletState


class UniformDropletGenerator:
    def __init__(self, coord_range=(0, 10), radii_range=(1, 100), num_particles=1, minimum_distance=0, *,
                 seed: int | None = None, periodic: bool = False, max_rounds: int = 1000, device=None):
        self.num_particles = num_particles
        self.coord_range = coord_range
        self.radii_range = radii_range
        self.minimum_distance = minimum_distance
        self.droplet_state = None
        self.seed = seed
        self.periodic = periodic
        self.max_rounds = max_rounds
        self.rounds = 0
        self._device = device

    def generate(self) -> DropletState:
        """uniform_droplet_generator.py:45-104."""
        n = int(self.num_particles)
        ctx = N.Context(max(n, 1), self._device)
        torch = ctx.torch
        seed = self.seed if self.seed is not None else int(np.random.SeedSequence().entropy % (1 << 64))
        pos = torch.empty((3, max(n, 1)), dtype=torch.float64, device=ctx.device)
        r = torch.empty(max(n, 1), dtype=torch.float64, device=ctx.device)
        self.rounds = ctx.generate_droplets(n, seed, self.coord_range[0], self.coord_range[1], self.radii_range[0],
                                            self.radii_range[1], self.minimum_distance, self.periodic,
                                            self.max_rounds, pos, r)
        positions = np.ascontiguousarray(pos[:, :n].T.cpu().numpy())
        self.droplet_state = DropletState(positions, r[:n].cpu().numpy(), 0)
        return self.droplet_state

    def print(self):
        if self.droplet_state is None:
            print("generate() the droplets first.")
            return
        for k, (p, rad) in enumerate(zip(self.droplet_state.positions, self.droplet_state.radii)):
            print(f"droplet {k}: position ({p[0]:.6g}, {p[1]:.6g}, {p[2]:.6g}), radius {rad:.6g}")

    def save(self, filename):
        """Excel file with columns X, Y, Z, Radius (uniform_droplet_generator.py:165-184)."""
        import pandas as pd

        if self.droplet_state is None:
            print("generate() the droplets first.")
            return
        p, r = self.droplet_state.positions, self.droplet_state.radii
        pd.DataFrame({"X": p[:, 0], "Y": p[:, 1], "Z": p[:, 2], "Radius": r}).to_excel(filename, index=False)

    def load(self, filename):
        import pandas as pd

        df = pd.read_excel(filename)
        positions = np.array(df[["X", "Y", "Z"]])
        self.num_particles = len(positions)
        self.droplet_state = DropletState(positions, np.array(df["Radius"]), 0)
