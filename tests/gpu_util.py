"""Helpers shared by the GPU tests."""

from __future__ import annotations

import numpy as np

import oracle as O

ETA_OIL = 0.06


def lognormal_state(n, seed=0, periodic=True, volume_fraction=0.02):
    from dem.particle_generator import LognormalDropletGenerator

    g = LognormalDropletGenerator(n, seed=seed, periodic=periodic, volume_fraction=volume_fraction)
    s = g.generate()
    return s.positions, s.radii, g.L


def consts():
    return O.physics_constants(eps_oil=2.85, eta_oil=ETA_OIL, eta_water=0.001, E=3e5)


def rel_norm(a, b):
    """Norm-wise relative error ||a - b|| / ||b||."""
    return float(np.linalg.norm(np.asarray(a) - b) / np.linalg.norm(b))


def ref_metric(a, b):
    """Per-droplet |a - b| / (|b| + 0.01 mean|b|): the error metric of the
    reference's benchmark (benchmarks/test.py:63-77).  Returns (mean, max)."""
    d = np.linalg.norm(np.asarray(a) - b, axis=1)
    nb = np.linalg.norm(b, axis=1)
    e = d / (nb + 0.01 * nb.mean())
    return float(e.mean()), float(e.max())
