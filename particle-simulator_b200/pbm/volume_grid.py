"""Volume classes of the population balance.

Drop-in for pbm/volume_grid.py:11-120 of ddkx21/particle-simulator: n_bins
classes between v_min and v_max with geometric, logarithmic or linear edges;
a volume belongs to the class whose left edge is the last one not above it,
and volumes outside [v_min, v_max] are clamped into the first or last class
(with one warning each way, as in the reference).
"""

from __future__ import annotations

import logging

import numpy as np

logger = logging.getLogger(__name__)


class VolumeGrid:
    def __init__(self, v_min: float, v_max: float, n_bins: int, spacing: str = "geometric") -> None:
        if v_min <= 0 or v_max <= v_min:
            raise ValueError("need 0 < v_min < v_max")
        if n_bins < 2:
            raise ValueError("need n_bins >= 2")
        self.n_bins = n_bins
        self.spacing = spacing
        if spacing == "geometric":
            self.edges = np.geomspace(v_min, v_max, n_bins + 1)
        elif spacing == "logarithmic":
            self.edges = 10 ** np.linspace(np.log10(v_min), np.log10(v_max), n_bins + 1)
        elif spacing == "linear":
            self.edges = np.linspace(v_min, v_max, n_bins + 1)
        else:
            raise ValueError(f"unknown spacing: {spacing}")
        lo, hi = self.edges[:-1], self.edges[1:]
        self.centers = np.sqrt(lo * hi) if spacing in ("geometric", "logarithmic") else 0.5 * (lo + hi)
        self.widths = np.diff(self.edges)
        self._warned_low = self._warned_high = False

    @classmethod
    def from_radii_range(cls, r_min: float, r_max: float, n_bins: int, spacing: str = "geometric") -> "VolumeGrid":
        return cls((4.0 / 3.0) * np.pi * r_min**3, (4.0 / 3.0) * np.pi * r_max**3, n_bins, spacing)

    def _warn(self, low: int, high: int):
        if high and not self._warned_high:
            logger.warning("VolumeGrid: %d volumes above v_max=%.3e clamped into class %d", high, self.edges[-1],
                           self.n_bins - 1)
            self._warned_high = True
        if low and not self._warned_low:
            logger.warning("VolumeGrid: %d volumes below v_min=%.3e clamped into class 0", low, self.edges[0])
            self._warned_low = True

    def bin_index(self, volume: float) -> int:
        raw = int(np.searchsorted(self.edges, volume, side="right")) - 1
        self._warn(int(raw < 0), int(raw >= self.n_bins))
        return max(0, min(raw, self.n_bins - 1))

    def bin_indices(self, volumes) -> np.ndarray:
        raw = np.searchsorted(self.edges, volumes, side="right").astype(np.intp) - 1
        self._warn(int(np.sum(raw < 0)), int(np.sum(raw >= self.n_bins)))
        np.clip(raw, 0, self.n_bins - 1, out=raw)
        return raw
