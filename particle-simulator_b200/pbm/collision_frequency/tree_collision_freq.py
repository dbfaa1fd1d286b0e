"""Collision counts between volume classes over the flat octree, on the B200.

Drop-in for pbm/collision_frequency/tree_collision_freq.py:14-175 of
ddkx21/particle-simulator: bound to a built ``FlatOctree``; ``compute`` counts
the touching pairs (|MIC(x_j - x_i)| <= r_i + r_j, each pair once) into an
(n_bins, n_bins) matrix, symmetric, with the tree walk of csrc/tree.cu
(``dem_tree_collision_matrix``) on the tree's own droplets.  The walk prunes
nodes with the reference's box distance; in periodic boxes that rule
over-estimates the distance to boxes across the boundary, so, like the
reference, it can miss contacts that ``DirectCollisionFrequency`` counts.
"""

from __future__ import annotations

import numpy as np


class TreeCollisionFrequency:
    def __init__(self, flat_tree, grid, max_particles: int) -> None:
        self.tree = flat_tree
        self.grid = grid
        self.n_bins = grid.n_bins
        self.max_particles = max_particles
        ctx = flat_tree._ctx
        torch = ctx.torch
        self._bins = torch.empty(max(int(max_particles), 1), dtype=torch.int32, device=ctx.device)
        self._matrix = torch.empty((self.n_bins, self.n_bins), dtype=torch.int32, device=ctx.device)

    def compute(self, positions, radii) -> np.ndarray:
        """Bins from the radii (grid.bin_indices of the volumes), counts from the
        droplets the tree was built on (tree_collision_freq.py:43-56)."""
        torch = self.tree._ctx.torch
        radii = np.asarray(radii, dtype=np.float64)
        n = len(radii)
        bins = np.ascontiguousarray(self.grid.bin_indices((4.0 / 3.0) * np.pi * radii**3), dtype=np.int32)
        if n > self._bins.numel():
            self._bins = torch.empty(n, dtype=torch.int32, device=self._bins.device)
        self._bins[:n].copy_(torch.from_numpy(bins))
        self.tree._tree.collision_matrix(self._bins, self.n_bins, self._matrix)
        return self._matrix.cpu().numpy().view(np.uint32).astype(np.float64)
