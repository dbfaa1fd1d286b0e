"""Collision counts between volume classes from all touching pairs, on the B200.

Drop-in for pbm/collision_frequency/direct_collision_freq.py:9-41 of
ddkx21/particle-simulator.  The reference loops over all N(N-1)/2 pairs;
here the touching pairs (|MIC(x_j - x_i)| <= r_i + r_j) come from the spatial
hash detection (csrc/hash.cu, the pair set of the collision detector) and are
binned on the device (``dem_pair_bin_matrix``).
"""

from __future__ import annotations

import numpy as np


class DirectCollisionFrequency:
    def __init__(self, grid, *, device=None) -> None:
        self.grid = grid
        self._device = device
        self._det = None

    def compute(self, positions, radii, L: float = 0.0, periodic: bool = False) -> np.ndarray:
        from dem.collision_detector import SpatialHashCollisionDetector

        radii = np.asarray(radii, dtype=np.float64)
        n = len(radii)
        nb = self.grid.n_bins
        if n < 2:
            return np.zeros((nb, nb))
        positions = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
        use_periodic = bool(periodic and L > 0)
        box = float(L) if L > 0 else float(np.ptp(positions, axis=0).max()) + 2.0 * float(radii.max()) + 1e-300
        if not use_periodic:  # open box: coordinates from the lower corner of the droplets
            positions = positions - positions.min(axis=0)
        if self._det is None:  # the detector grows its workspace with n
            self._det = SpatialHashCollisionDetector(num_particles=n, L=box, device=self._device)
        det = self._det
        torch = det._ctx.torch
        st, _ = det._io.positions(positions, radii)
        k, pairs, counts = det.detect_device(n, st.pos, st.r, box, use_periodic)
        bins = np.ascontiguousarray(self.grid.bin_indices((4.0 / 3.0) * np.pi * radii**3), dtype=np.int32)
        bins_d = torch.from_numpy(bins).to(det._ctx.device)
        out = torch.empty((nb, nb), dtype=torch.int32, device=det._ctx.device)
        det._ctx.pair_bin_matrix(pairs, counts, k, bins_d, nb, out)
        return out.cpu().numpy().view(np.uint32).astype(np.float64)
