"""Spatial-hash collision detection on the B200.

Drop-in for dem/collision_detector/spatial_hash_collision_detector.py:27-316
of ddkx21/particle-simulator.  The hash table size is fixed by the
constructor (next power of two >= 2 * num_particles, :42), the cell size is
2 max r and the grid max(1, ceil(L / cell)) (:256-262), and the pair set is
bit-identical to the reference's ``np.unique`` output (csrc/hash.cu).

Differences from the reference, all on inputs where the reference misbehaves:
* every colliding pair is returned (the reference silently drops hits beyond
  a buffer of ``num_particles`` entries, :227-229);
* inputs longer than ``num_particles`` grow the workspace (the reference
  truncates them but still loops over all of them, :268-282).
"""

from __future__ import annotations

import numpy as np

from .. import _native as N
from .._io import Stager
from .collision_detector_base import CollisionDetector

_EMPTY_PAIRS = np.empty((0, 2), dtype=np.int32)


def _next_power_of_2(n: int) -> int:
    """Smallest power of two >= n (spatial_hash_collision_detector.py:18-23)."""
    p = 1
    while p < n:
        p <<= 1
    return p


class SpatialHashCollisionDetector(CollisionDetector):
    def __init__(self, num_particles: int, L: float = 1.0, boundary_mode: str = "periodic", *, device=None):
        self._max_particles = num_particles
        self._L = L
        self._boundary_mode = boundary_mode
        self._hash_table_size = _next_power_of_2(2 * num_particles)
        self._hash_mask = self._hash_table_size - 1
        self._ctx = N.Context(max(int(num_particles), 1), device)
        self._io = Stager(self._ctx)
        self._pair_capacity = max(4 * int(num_particles), 1024)
        torch = self._ctx.torch
        self._pairs = torch.empty((self._pair_capacity, 2), dtype=torch.int32, device=self._ctx.device)
        self._counts = torch.zeros(2, dtype=torch.int64, device=self._ctx.device)
        self._counts_host = torch.zeros(2, dtype=torch.int64, pin_memory=True)

    def _reserve(self, n):
        if n > self._ctx.capacity:
            self._ctx.reserve(n)

    def detect_device(self, n, pos_soa, r, L, periodic):
        """Device-resident detection: returns (K, pairs view (K, 2) int32 on the device).

        Reads the pair count back (a 16-byte synchronising copy); grows the pair
        buffer and re-runs when it overflows."""
        torch = self._ctx.torch
        self._reserve(n)
        while True:
            self._ctx.hash_detect(n, pos_soa, r, L, periodic, self._hash_table_size, self._pairs,
                                  self._pair_capacity, self._counts)
            self._counts_host.copy_(self._counts, non_blocking=True)
            torch.cuda.current_stream(self._ctx.device).synchronize()
            k = int(self._counts_host[0])
            if k <= self._pair_capacity:
                break
            self._ctx.device_errors()  # clear the overflow flag, then retry with room for every pair
            self._pair_capacity = _next_power_of_2(k)
            self._pairs = torch.empty((self._pair_capacity, 2), dtype=torch.int32, device=self._ctx.device)
        return k, self._pairs[:k], self._counts

    def detect_launch(self, n, pos_soa, r, L, periodic):
        """The detection kernels and an asynchronous copy of the pair count into
        pinned host memory, without synchronising (capturable in a CUDA graph).
        Read the result with ``detect_finish`` once the stream has synchronised."""
        self._reserve(n)
        self._ctx.hash_detect(n, pos_soa, r, L, periodic, self._hash_table_size, self._pairs, self._pair_capacity,
                              self._counts)
        self._counts_host.copy_(self._counts, non_blocking=True)

    def detect_finish(self, n, pos_soa, r, L, periodic):
        """(K, pairs, counts) of the last ``detect_launch``; on a pair-buffer
        overflow the detection runs again with room for every pair (the buffer
        is then a new allocation)."""
        k = int(self._counts_host[0])
        if k <= self._pair_capacity:
            return k, self._pairs[:k], self._counts
        return self.detect_device(n, pos_soa, r, L, periodic)

    def detect(self, positions, radii, *, L: float | None = None, boundary_mode: str | None = None):
        """(is_collision, pairs (K, 2) int32), spatial_hash_collision_detector.py:233-316."""
        use_L = L if L is not None else self._L
        use_boundary = boundary_mode if boundary_mode is not None else self._boundary_mode
        n = len(radii)
        if n == 0:
            return False, _EMPTY_PAIRS.copy()
        self._reserve(n)
        st, on_dev = self._io.positions(positions, radii)
        k, pairs, _ = self.detect_device(st.n, st.pos, st.r, float(use_L), use_boundary == "periodic")
        if k == 0:
            return False, (pairs.clone() if on_dev else _EMPTY_PAIRS.copy())
        if on_dev:
            return True, pairs.clone()
        h = self._io.buf.host("pairs_h", (k, 2), dtype=self._ctx.torch.int32)
        h.copy_(pairs)
        return True, h.numpy().copy()
