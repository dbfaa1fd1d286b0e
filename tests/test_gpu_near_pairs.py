"""Near pairs in dense clusters: the mixed symmetric pass on Morton-ordered
blocks against the FP64 drop-in (bit-exact with the oracle).

The pass evaluates near-contact pairs (|d| <= k (r_i + r_j)) in FP64 from a
per-warp queue.  In the seeded lognormal states a warp meets a few of them per
block pair; here clusters of 512 droplets at ~11 % and ~3 % local volume
fraction (some of them wrapped across the periodic faces) put hundreds of
near pairs into one block pair.  The queue is then evaluated while a j
sub-tile is running (its j-side terms collect for that sub-tile) and after
sub-tiles have written their partial sums (the terms are added onto them), in
diagonal and off-diagonal block pairs.  Reference formulas:
direct_droplet_force_calculator.py:183-253 (forces) and :354-411 (Oseen).
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from gpu_util import ETA_OIL, consts, ref_metric, rel_norm

pytestmark = pytest.mark.gpu

N = 16384
# the bounds of the measured configurations: forces 1e-5 against FP64 (norm-wise
# and per droplet); velocities carry the Oseen sum's cancellation, so their
# per-droplet bound is wider.  Measured on a B200: forces 2.1e-8 / 3.4e-6,
# velocities 6.9e-7 / 5.8e-5.
FORCE_NORM_TOL = 1e-5
FORCE_PER_DROPLET_TOL = 1e-5
VEL_NORM_TOL = 1e-5
VEL_PER_DROPLET_TOL = 5e-4


def clustered_state(seed=0):
    """8 clusters of 512 droplets (4 of radius 100 um, 4 of 300 um) in a
    uniform background at ~1 % volume fraction, periodic box."""
    rng = np.random.default_rng(seed)
    r = np.clip(5e-6 * np.exp(0.35 * rng.standard_normal(N)), 1e-6, 30e-6)
    L = float(np.cbrt(N * np.mean(4.0 / 3.0 * np.pi * r**3) / 0.01))
    pos = rng.uniform(0.0, L, size=(N, 3))
    centres = rng.uniform(0.0, L, size=(8, 3))
    centres[0] = [0.02 * L, 0.5 * L, 0.99 * L]  # wraps across two faces
    for c in range(8):
        rad = 100e-6 if c < 4 else 300e-6
        d = rng.standard_normal((512, 3))
        d *= (rad * np.cbrt(rng.uniform(0.0, 1.0, 512)) / np.linalg.norm(d, axis=1))[:, None]
        pos[c * 512:(c + 1) * 512] = centres[c] + d
    return np.mod(pos, L), r, L


def test_clustered_near_pairs_mixed_against_fp64():
    from dem.force_calculator import DirectDropletForceCalculator

    pos, r, L = clustered_state()
    kw = dict(num_particles=N, eta_oil=ETA_OIL, L=L, boundary_mode="periodic")
    mixed = DirectDropletForceCalculator(precision="mixed", **kw)
    plan = mixed._ctx.plan(N)
    assert plan["schedule"] == "symmetric" and plan["i_per_thread"] == 4, plan
    exact = DirectDropletForceCalculator(precision="fp64", **kw)
    F, V = mixed.calculate_forces_and_convection(pos, r)
    F64 = exact.calculate(pos, r)
    V64 = exact.calculate_convection(pos, r, F)  # the same forces in: the convection pass alone
    Vm = mixed.calculate_convection(pos, r, F)
    ef, ev = rel_norm(F, F64), rel_norm(Vm, V64)
    mf, mv = ref_metric(F, F64)[1], ref_metric(Vm, V64)[1]
    msg = f"forces {ef:.2e} / {mf:.2e} per droplet, velocities {ev:.2e} / {mv:.2e}"
    assert ef <= FORCE_NORM_TOL and mf <= FORCE_PER_DROPLET_TOL, msg
    assert ev <= VEL_NORM_TOL and mv <= VEL_PER_DROPLET_TOL, msg
    # the FP64 path is the oracle's sum, bit for bit; check it on the first cluster's rows
    m, eta, _ = consts()
    F_or = O.direct_forces(pos, r, m, L, True, rows=(0, 512))[:512]
    assert np.array_equal(F64[:512], F_or)
    # deterministic: the queue's order depends only on the inputs
    F2, V2 = mixed.calculate_forces_and_convection(pos, r)
    assert np.array_equal(F, F2) and np.array_equal(V, V2)
    assert mixed._ctx.device_errors() == 0
