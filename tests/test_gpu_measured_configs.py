"""The measured configurations themselves, at full size, against the oracle.

* Direct DEM at N = 65,536 (and a ragged 65,000), mixed precision with the
  automatic schedule (symmetric blocks, 4 rows per thread): forces on three row
  samples (the first 1,024 rows, one whole block row in the middle, the last
  block) against the oracle's FP64 sum over all columns
  (direct_droplet_force_calculator.py:202-253), and the plain Oseen
  convection of the oracle's own forces on the same rows
  (direct_droplet_force_calculator.py:354-411).
* Barnes-Hut on Morton keys at N = 2^20, theta = 0.5, leaf 16, with the
  reference's acceptance rule only (window 0: s^2 < theta^2 D^2 at the
  centre's minimum image, flat_tree.py:871): forces on a seeded 4,096-droplet
  subsample against the oracle's direct FP64 sum over all 2^20 droplets.
* The adjoint at N = 16,384, 200 Euler steps, a checkpoint every 20 steps, in
  the open box: gradients with respect to 32 seeded initial coordinates against
  FP64 central differences (h = 1e-9 m).  In a periodic box at this size pair
  separations cross L/2 during the run and the minimum image jumps, so central
  differences there measure a staircase, not the derivative.
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from gpu_util import ETA_OIL, consts, lognormal_state, ref_metric, rel_norm

pytestmark = pytest.mark.gpu

# forces: the north star's bound is 1e-5 relative against FP64; velocities carry
# the Oseen sum's cancellation (sum_j F_j = 0), so their bound is wider
FORCE_NORM_TOL = 1e-5
FORCE_PER_DROPLET_TOL = 1e-5
VEL_NORM_TOL = 1e-5
VEL_PER_DROPLET_TOL = 5e-4


def _row_samples(n, block):
    mid = (n // block // 2) * block
    last = ((n - 1) // block) * block
    return [(0, 1024), (mid, mid + block), (last, n)]


@pytest.mark.parametrize("n", [65536, 65000])
def test_config1_mixed_auto_schedule_against_oracle(n):
    from dem.force_calculator import DirectDropletForceCalculator

    pos, r, L = lognormal_state(n, seed=0)
    m, eta, _ = consts()
    fc = DirectDropletForceCalculator(num_particles=n, eta_oil=ETA_OIL, L=L, boundary_mode="periodic",
                                      precision="mixed")
    plan = fc._ctx.plan(n)
    assert plan["schedule"] == "symmetric" and plan["i_per_thread"] == 4, plan
    block = plan["threads"] * plan["i_per_thread"]
    F, V = fc.calculate_forces_and_convection(pos, r)
    F_ref = O.direct_forces(pos, r, m, L, True)  # every row: the convection below needs all forces
    V_of_ref = fc.calculate_convection(pos, r, F_ref)  # the mixed Oseen pass alone, on the oracle's forces
    for i0, i1 in _row_samples(n, block):
        V_ref = O.direct_convection(pos, F_ref, eta, L, True, rows=(i0, i1))[i0:i1]
        assert rel_norm(F[i0:i1], F_ref[i0:i1]) <= FORCE_NORM_TOL, (i0, i1)
        assert ref_metric(F[i0:i1], F_ref[i0:i1])[1] <= FORCE_PER_DROPLET_TOL, (i0, i1)
        assert rel_norm(V_of_ref[i0:i1], V_ref) <= VEL_NORM_TOL, (i0, i1)
        assert ref_metric(V_of_ref[i0:i1], V_ref)[1] <= VEL_PER_DROPLET_TOL, (i0, i1)
        # the fused call: its convection takes the mixed forces, so it carries both passes' errors
        assert rel_norm(V[i0:i1], V_ref) <= VEL_NORM_TOL, (i0, i1)
    assert rel_norm(F, F_ref) <= FORCE_NORM_TOL
    assert fc._ctx.device_errors() == 0


def test_config2_barnes_hut_2p20_reference_rule_within_1e_3():
    from dem.octree import MortonTreeForceCalculator

    n = 1 << 20
    pos, r, L = lognormal_state(n, seed=0)
    m, _, _ = consts()
    tc = MortonTreeForceCalculator(num_particles=n, theta=0.5, mpl=16, eta_oil=ETA_OIL, L=L, periodic=True,
                                   window_level=0)
    F = tc.calculate(pos, r)
    st = tc.stats()
    assert st["levels"] >= 6 and st["node_terms"] > 0
    sample = np.sort(np.random.default_rng(4096).choice(n, 4096, replace=False))
    # the oracle sums rows 0..k-1; put the sample first (the column order only moves FP64 rounding)
    perm = np.concatenate([sample, np.setdiff1d(np.arange(n), sample)])
    F_ref = O.direct_forces(pos[perm], r[perm], m, L, True, rows=(0, len(sample)))[: len(sample)]
    err = rel_norm(F[sample], F_ref)
    mean_metric = ref_metric(F[sample], F_ref)[0]
    assert err <= 1e-3, err
    assert mean_metric <= 1e-3, mean_metric
    assert tc._ctx.device_errors() == 0


def test_config4_adjoint_open_box_n16384_against_central_differences():
    import torch

    from dem.adjoint import DirectTrajectory, mean_squared_z_displacement, pair_softplus

    n, steps, dt = 16384, 200, 1e-4
    pos, r, L = lognormal_state(n, seed=0)
    x0 = torch.tensor(pos, dtype=torch.float64, device="cuda")
    rr = torch.tensor(r, dtype=torch.float64, device="cuda")
    E = torch.tensor(3e5, dtype=torch.float64, device="cuda")
    sim = DirectTrajectory(L, steps, dt, checkpoint_every=20, precision="fp64", eta_oil=ETA_OIL, eta_water=0.001,
                           eps_oil=2.85, boundary_mode="open")

    def loss_of(x):
        xT, D = sim(x, rr, E)
        return mean_squared_z_displacement(D) + pair_softplus(xT, rr, L, periodic=False)

    xg = x0.clone().requires_grad_()
    (gx,) = torch.autograd.grad(loss_of(xg), (xg,))
    rng = np.random.default_rng(7)
    fd, ad = [], []
    with torch.no_grad():
        for i, c in zip(rng.integers(0, n, 32), rng.integers(0, 3, 32)):
            h = 1e-9
            xp, xm = x0.clone(), x0.clone()
            xp[i, c] += h
            xm[i, c] -= h
            fd.append(float(loss_of(xp) - loss_of(xm)) / (2 * h))
            ad.append(float(gx[i, c]))
    fd, ad = np.array(fd), np.array(ad)
    assert np.linalg.norm(fd - ad) / np.linalg.norm(fd) <= 1e-6
    assert np.abs(fd - ad).max() <= 1e-6 * np.abs(fd).max()
