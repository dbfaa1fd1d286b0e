"""Ensembles of independent boxes (main_multi.py-style) on the GPU.

Per box, the batched passes must be bit-identical to the single-box
mixed-precision calls (symmetric schedule, same block size), and within the
mixed-precision tolerances of the FP64 oracle.  Eager steps and CUDA-graph
replays must agree bit for bit; the autotuner must leave a valid tiling whose
results equal any other grid shape at the same block size."""

from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from gpu_util import ETA_OIL, consts, lognormal_state, rel_norm

pytestmark = pytest.mark.gpu

MIXED_NORM_TOL = 1e-6
MIXED_V_NORM_TOL = 2e-6

SIZES = [300, 1000, 37, 0, 2049, 513]


def _states(sizes=SIZES, seed=11):
    states, Ls = [], []
    for k, n in enumerate(sizes):
        if n == 0:
            states.append((np.zeros((0, 3)), np.zeros(0)))
            Ls.append(4e-4)
            continue
        pos, r, L = lognormal_state(n, seed=seed + k)
        states.append((pos, r))
        Ls.append(L)
    return states, np.array(Ls)


def _ensemble(states, Ls, **kw):
    from dem.ensemble import DropletEnsemble

    return DropletEnsemble(states, Ls, eta_oil=ETA_OIL, **kw)


def _single(n, L):
    from dem.force_calculator import DirectDropletForceCalculator

    fc = DirectDropletForceCalculator(num_particles=max(n, 1), eta_oil=ETA_OIL, L=L, precision="mixed")
    fc.set_tuning(i_per_thread=4, schedule="symmetric")
    return fc


@pytest.mark.parametrize("ipt,ctas", [(4, 0), (2, 0), (4, 150), (2, 7)])
def test_batched_equals_single_box_and_oracle(ipt, ctas):
    states, Ls = _states()
    ens = _ensemble(states, Ls)
    ens.set_tuning(ipt, ctas)
    out = ens.forces_and_convection()
    m, eta, _ = consts()
    for (pos, r), L, (F, V) in zip(states, Ls, out):
        if len(r) == 0:
            assert F.shape == (0, 3)
            continue
        fc = _single(len(r), L)
        fc.set_tuning(i_per_thread=ipt)
        F1, V1 = fc.calculate_forces_and_convection(pos, r)
        np.testing.assert_array_equal(F, F1)
        np.testing.assert_array_equal(V, V1)
        F_ref = O.direct_forces(pos, r, m, L, True)
        assert rel_norm(F, F_ref) <= MIXED_NORM_TOL
        assert rel_norm(V, O.direct_convection(pos, F_ref, eta, L, True)) <= MIXED_V_NORM_TOL
    assert ens.ctx.device_errors() == 0


def test_grid_shape_does_not_change_results():
    states, Ls = _states([700, 1500, 260], seed=3)
    ens = _ensemble(states, Ls)
    ens.set_tuning(4, 0)
    a = ens.forces_and_convection()
    for ctas in (1, 3, 148, 1000):
        ens.set_tuning(4, ctas)
        b = ens.forces_and_convection()
        for (F, V), (F2, V2) in zip(a, b):
            np.testing.assert_array_equal(F, F2)
            np.testing.assert_array_equal(V, V2)


def test_step_matches_oracle_euler_per_box():
    states, Ls = _states([400, 900], seed=5)
    ens = _ensemble(states, Ls)
    dt = 1e-4
    ens.step(dt, steps=1)
    F_dev, V_dev = ens.F.T.cpu().numpy(), ens.V.T.cpu().numpy()
    _, _, sf = consts()
    for b, ((pos, r), L) in enumerate(zip(states, Ls)):
        s = ens.box_slice(b)
        want = O.euler_direct(pos, r, F_dev[s], V_dev[s], sf, dt, L, True)
        np.testing.assert_array_equal(ens.positions()[b], want)


def test_graph_replay_equals_eager_and_sequential():
    states, Ls = _states([333, 1200, 0, 77], seed=8)
    dt = 1e-4
    eager = _ensemble(states, Ls)
    eager.step(dt, steps=4)
    graph = _ensemble(states, Ls)
    from dem._native import launch_count

    graph.step(dt, steps=1, graph=True)  # capture + 1 replay
    c0 = launch_count()
    graph.step(dt, steps=3, graph=True)
    assert launch_count() - c0 >= 3 * 10  # kernels of the replayed graph are counted
    for a, b in zip(eager.positions(), graph.positions()):
        np.testing.assert_array_equal(a, b)
    seq = _ensemble(states, Ls)
    seq.ctx.set_tuning(i_per_thread=4, schedule="symmetric")
    seq.step_sequential(dt, steps=4)
    for a, b in zip(eager.positions(), seq.positions()):
        np.testing.assert_array_equal(a, b)


def test_autotune_picks_a_candidate_and_keeps_results():
    states, Ls = _states([2000, 3000, 1024], seed=9)
    ens = _ensemble(states, Ls)
    res = ens.autotune(reps=1)
    assert res["i_per_thread"] in (2, 4) and res["ctas"] >= 0 and res["ms"] > 0
    F, V = ens.compute()
    m, eta, _ = consts()
    Fh = F.T.cpu().numpy()
    for b, ((pos, r), L) in enumerate(zip(states, Ls)):
        F_ref = O.direct_forces(pos, r, m, L, True)
        assert rel_norm(Fh[ens.box_slice(b)], F_ref) <= MIXED_NORM_TOL


def test_rejects_bad_tables():
    from dem import _native as N

    ctx = N.Context(16)
    with pytest.raises(ValueError):
        N.Batch(ctx, [0, 5, 3], [1.0, 1.0], True)  # decreasing offsets
    with pytest.raises(ValueError):
        N.Batch(ctx, [0, 5], [0.0], True)  # non-positive side
    b = N.Batch(ctx, [0, 5], [1.0], True)
    with pytest.raises(ValueError):
        b.set_tuning(3, 0)
