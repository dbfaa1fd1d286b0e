"""Direct O(N^2) force and convection on the GPU against the oracle.

FP64 (the reference drop-in): bit-exact.
Mixed precision: forces within 1e-6 norm-wise and 1e-5 per droplet
(reference benchmark metric); convection velocities within 2e-6 norm-wise and
5e-5 per droplet.  The Oseen sum cancels strongly (sum_j F_j = 0; its
condition number reaches ~3e3 per droplet), so FP32 pair terms leave a larger
relative error on the velocities than on the forces."""

from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN
from gpu_util import ETA_OIL, consts, lognormal_state, ref_metric, rel_norm

pytestmark = pytest.mark.gpu

MIXED_NORM_TOL = 1e-6
MIXED_PER_DROPLET_TOL = 1e-5
MIXED_V_NORM_TOL = 2e-6
MIXED_V_PER_DROPLET_TOL = 5e-5


def _calc(n, L, periodic=True, precision="fp64", eta_oil=ETA_OIL):
    from dem.force_calculator import DirectDropletForceCalculator

    return DirectDropletForceCalculator(num_particles=n, eta_oil=eta_oil, L=L,
                                        boundary_mode="periodic" if periodic else "open", precision=precision)


@pytest.mark.parametrize("name", sorted(p.name for p in GOLDEN.glob("direct_*.npz")))
def test_fp64_bit_exact_against_golden(golden, name):
    g = golden(name)
    fc = _calc(len(g["radii"]), float(g["L"]), bool(g["periodic"]), eta_oil=float(g["eta_oil"]))
    F, V = fc.calculate_forces_and_convection(g["positions"], g["radii"])
    np.testing.assert_array_equal(F, g["forces"])
    np.testing.assert_array_equal(V, g["velocities"])
    np.testing.assert_array_equal(fc.calculate(g["positions"], g["radii"]), g["forces"])
    np.testing.assert_array_equal(fc.calculate_convection(g["positions"], g["radii"], g["forces"]), g["velocities"])


@pytest.mark.parametrize("periodic", [True, False])
def test_fp64_bit_exact_lognormal_2000(periodic):
    pos, r, L = lognormal_state(2000, seed=0, periodic=periodic)
    m, eta, _ = consts()
    F, V = _calc(2000, L, periodic).calculate_forces_and_convection(pos, r)
    F_ref = O.direct_forces(pos, r, m, L, periodic)
    np.testing.assert_array_equal(F, F_ref)
    np.testing.assert_array_equal(V, O.direct_convection(pos, F_ref, eta, L, periodic))


def test_fp64_torch_tensors_stay_on_device():
    import torch

    pos, r, L = lognormal_state(700, seed=4)
    m, eta, _ = consts()
    fc = _calc(700, L)
    F, V = fc.calculate_forces_and_convection(torch.as_tensor(pos, device="cuda"), torch.as_tensor(r, device="cuda"))
    assert F.is_cuda and V.is_cuda and F.shape == (700, 3)
    F_ref = O.direct_forces(pos, r, m, L, True)
    np.testing.assert_array_equal(F.cpu().numpy(), F_ref)
    np.testing.assert_array_equal(V.cpu().numpy(), O.direct_convection(pos, F_ref, eta, L, True))


@pytest.mark.parametrize("n,seed", [(2000, 0), (8192, 1)])
def test_mixed_against_fp64_oracle(n, seed):
    pos, r, L = lognormal_state(n, seed=seed)
    m, eta, _ = consts()
    F, V = _calc(n, L, precision="mixed").calculate_forces_and_convection(pos, r)
    F_ref = O.direct_forces(pos, r, m, L, True)
    V_ref = O.direct_convection(pos, F_ref, eta, L, True)
    assert rel_norm(F, F_ref) <= MIXED_NORM_TOL
    assert rel_norm(V, V_ref) <= MIXED_V_NORM_TOL
    assert ref_metric(F, F_ref)[1] <= MIXED_PER_DROPLET_TOL
    assert ref_metric(V, V_ref)[1] <= MIXED_V_PER_DROPLET_TOL


@pytest.mark.parametrize("ipt,threads,splits,schedule", [
    (1, 128, 0, "split"), (2, 256, 3, "split"), (4, 64, 1, "split"), (8, 128, 0, "split"), (4, 512, 7, "split"),
    (1, 0, 0, "symmetric"), (2, 0, 0, "symmetric"), (4, 0, 0, "symmetric"),
    (2, 0, 0, "symmetric_plain"), (4, 0, 0, "symmetric_plain"),
])
def test_mixed_tunings_agree_and_are_deterministic(ipt, threads, splits, schedule):
    pos, r, L = lognormal_state(3000, seed=2)
    m, eta, _ = consts()
    fc = _calc(3000, L, precision="mixed")
    fc.set_tuning(i_per_thread=ipt, threads=threads, j_splits=splits, schedule=schedule)
    F1, V1 = fc.calculate_forces_and_convection(pos, r)
    F2, V2 = fc.calculate_forces_and_convection(pos, r)
    np.testing.assert_array_equal(F1, F2)
    np.testing.assert_array_equal(V1, V2)
    F_ref = O.direct_forces(pos, r, m, L, True)
    assert rel_norm(F1, F_ref) <= MIXED_NORM_TOL
    assert rel_norm(V1, O.direct_convection(pos, F_ref, eta, L, True)) <= MIXED_V_NORM_TOL


@pytest.mark.parametrize("periodic,n", [(True, 20000), (False, 16384)])
def test_symmetric_morton_blocks_against_oracle_and_plain_blocks(periodic, n):
    """The symmetric schedule on Morton-ordered blocks (fast, medium and slow
    j lists) against the oracle, and against the same schedule on blocks in
    the caller's order: the same pairs go to FP64 in both, only the FP32
    summation order differs."""
    pos, r, L = lognormal_state(n, seed=11, periodic=periodic)
    m, eta, _ = consts()
    fc = _calc(n, L, periodic, precision="mixed")
    fc.set_tuning(schedule="symmetric")
    assert fc._ctx.plan(n, periodic)["schedule"] == "symmetric"
    F, V = fc.calculate_forces_and_convection(pos, r)
    F2, V2 = fc.calculate_forces_and_convection(pos, r)
    np.testing.assert_array_equal(F, F2)  # deterministic
    np.testing.assert_array_equal(V, V2)
    rows = (0, 2048)
    F_ref = O.direct_forces(pos, r, m, L, periodic)
    V_ref = O.direct_convection(pos, F_ref, eta, L, periodic, rows=rows)[: rows[1]]
    assert rel_norm(F, F_ref) <= MIXED_NORM_TOL
    assert ref_metric(F, F_ref)[1] <= MIXED_PER_DROPLET_TOL
    assert rel_norm(V[: rows[1]], V_ref) <= MIXED_V_NORM_TOL
    assert ref_metric(V[: rows[1]], V_ref)[1] <= MIXED_V_PER_DROPLET_TOL
    fc.set_tuning(schedule="symmetric_plain")
    assert fc._ctx.plan(n, periodic)["schedule"] == "symmetric_plain"
    Fp, Vp = fc.calculate_forces_and_convection(pos, r)
    assert rel_norm(F, Fp) <= MIXED_NORM_TOL
    assert rel_norm(V, Vp) <= MIXED_V_NORM_TOL
    assert fc._ctx.device_errors() == 0


@pytest.mark.parametrize("periodic,n,schedule", [(True, 20000, "symmetric"), (False, 9000, "symmetric"),
                                                  (True, 3000, "split"), (True, 5000, "symmetric_plain")])
def test_fused_call_equals_the_two_passes(periodic, n, schedule):
    """dem_direct_forces_and_convection (the convection pass reuses the force
    pass's Morton order) against dem_direct_forces + dem_direct_convection."""
    import torch

    pos, r, L = lognormal_state(n, seed=13, periodic=periodic)
    m, eta, _ = consts()
    fc = _calc(n, L, periodic, precision="mixed")
    fc.set_tuning(schedule=schedule)
    st, _ = fc._io.positions(pos, r)
    from dem import _native as N

    ctx, prec = fc._ctx, N.PREC_MIXED
    F1 = torch.empty((3, n), dtype=torch.float64, device="cuda")
    V1, F2, V2 = torch.empty_like(F1), torch.empty_like(F1), torch.empty_like(F1)
    ctx.direct_forces(n, st.pos, st.r, fc.m_const, L, periodic, prec, F1)
    ctx.direct_convection(n, st.pos, st.r, F1, fc.eta_const, L, periodic, prec, V1)
    ctx.direct_forces_and_convection(n, st.pos, st.r, fc.m_const, fc.eta_const, L, periodic, prec, F2, V2)
    assert torch.equal(F1, F2) and torch.equal(V1, V2)
    # and once more after a pass on other positions (the kept order must not leak into a later call)
    other, _, _ = lognormal_state(n, seed=14, periodic=periodic)
    st2, _ = fc._io.positions(other, r, tag="other")
    ctx.direct_forces(n, st2.pos, st.r, fc.m_const, L, periodic, prec, F1)
    ctx.direct_convection(n, st.pos, st.r, F2, fc.eta_const, L, periodic, prec, V1)
    assert torch.equal(V1, V2)
    assert ctx.device_errors() == 0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_open_boundary_and_contact_cut(golden, precision):
    g = golden("direct_contact_n48.npz")  # many pairs inside r_i + r_j
    fc = _calc(48, float(g["L"]), True, precision=precision)
    F, V = fc.calculate_forces_and_convection(g["positions"], g["radii"])
    assert rel_norm(F, g["forces"]) <= (0 if precision == "fp64" else MIXED_NORM_TOL)
    assert rel_norm(V, g["velocities"]) <= (0 if precision == "fp64" else MIXED_V_NORM_TOL)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_reference_invariants(precision):
    # tests/force_calculator/test_direct_droplet_force_calculator.py upstream
    from dem.force_calculator import DirectDropletForceCalculator

    fc = DirectDropletForceCalculator(num_particles=4, L=1.0, boundary_mode="open", precision=precision)
    f = fc.calculate(np.array([[0.5, 0.5, 0.5]]), np.array([1e-5]))
    assert f.shape == (1, 3)
    np.testing.assert_allclose(f[0], 0.0)
    f = fc.calculate(np.array([[0.4, 0.5, 0.5], [0.6, 0.5, 0.5]]), np.array([2e-5, 2e-5]))
    np.testing.assert_allclose(f[0], -f[1], rtol=1e-10)
    pos = np.array([[0.05, 0.5, 0.5], [0.95, 0.5, 0.5]])
    rr = np.array([1e-5, 1e-5])
    f_open = DirectDropletForceCalculator(num_particles=4, L=1.0, boundary_mode="open", precision=precision).calculate(pos, rr)
    f_per = DirectDropletForceCalculator(num_particles=4, L=1.0, boundary_mode="periodic", precision=precision).calculate(pos, rr)
    assert f_open[0, 0] * f_per[0, 0] < 0


def test_capacity_grows_and_zero_radii():
    fc = _calc(4, 1e-3)
    pos, r, L = lognormal_state(300, seed=7)
    fc.L = L
    m, eta, _ = consts()
    F = fc.calculate(pos, r)  # more droplets than the constructor capacity
    np.testing.assert_array_equal(F, O.direct_forces(pos, r, m, L, True))
    z = np.zeros(5)
    p = np.random.default_rng(0).uniform(0, L, (5, 3))
    for prec in ("fp64", "mixed"):
        fc2 = _calc(5, L, precision=prec)
        F0, V0 = fc2.calculate_forces_and_convection(p, z)
        assert np.all(F0 == 0) and np.all(np.isfinite(V0))


def test_euler_update_bit_exact():
    import torch

    pos, r, L = lognormal_state(1500, seed=5)
    m, eta, sf = consts()
    fc = _calc(1500, L)
    st, _ = fc._io.positions(pos, r)
    F, V = fc.forces_and_convection_soa(st.n, st.pos, st.r)
    out = torch.empty((3, st.n), dtype=torch.float64, device="cuda")
    fc._ctx.euler_update(st.n, st.pos, st.r, F, V, sf, 1e-3, L, True, out)
    got = fc._io.download([out], st.n)[0]
    F_ref = O.direct_forces(pos, r, m, L, True)
    V_ref = O.direct_convection(pos, F_ref, eta, L, True)
    np.testing.assert_array_equal(got, O.euler_direct(pos, r, F_ref, V_ref, sf, 1e-3, L, True))
    # wrap of positions pushed outside the box (numpy remainder semantics)
    shifted = pos.copy()
    shifted[:10] -= L * 1.5
    shifted[10:20] += L * 0.75
    st, _ = fc._io.positions(shifted, r)
    zero = torch.zeros((3, st.n), dtype=torch.float64, device="cuda")
    fc._ctx.euler_update(st.n, st.pos, st.r, zero, zero, sf, 1e-3, L, True, out)
    got = fc._io.download([out], st.n)[0]
    np.testing.assert_array_equal(got, np.mod(shifted, L))
    assert fc._ctx.device_errors() == 0


def test_plan_and_launch_counter():
    from dem._native import launch_count

    pos, r, L = lognormal_state(1000, seed=3)
    fc = _calc(1000, L, precision="mixed")
    assert fc._ctx.plan(65536)["schedule"] == "symmetric"
    assert fc._ctx.plan(100)["schedule"] == "split"  # auto: too small for block pairs
    # auto keeps >= 3.5 block pairs per SM (148 SMs): split up to ~4k, 2 rows per thread, then 4
    assert fc._ctx.plan(2000)["schedule"] == "split"
    assert (fc._ctx.plan(8192)["schedule"], fc._ctx.plan(8192)["i_per_thread"]) == ("symmetric", 2)
    assert (fc._ctx.plan(16384)["schedule"], fc._ctx.plan(16384)["i_per_thread"]) == ("symmetric", 4)
    fc.set_tuning(schedule="split")
    p = fc._ctx.plan(65536)
    assert p["schedule"] == "split" and p["j_splits"] >= 1 and p["ctas"] >= 148
    fc.set_tuning(schedule="auto")
    fc.calculate_forces_and_convection(pos, r)  # first call allocates
    c0 = launch_count()
    fc.calculate_forces_and_convection(pos, r)
    # forces: max, prep, pass, reduce; convection: 2 max, 2 prep, pass, reduce; plus the layout kernels
    assert launch_count() - c0 >= 10
