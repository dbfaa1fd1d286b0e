"""The periodic-image Oseen correction on the GPU (csrc/corr.cu, the fused FP64
convection of csrc/direct_fp64.cu, the tree walks of csrc/tree.cu and
csrc/bh.cu) through the drop-in classes, against the reference's own outputs
(tests/golden/corr_*.npz) and the oracle's restatement at larger sizes.

* FP64 direct and the FP64 parity tree: bit-identical;
* mixed direct (FP32 correction pass): norm-wise relative velocity error
  <= 1e-5 and every droplet's error <= 1e-5 of the mean |V|.  The correction
  sum over j cancels to ~1e-3 of the sum of its |terms| (the forces sum to
  zero), and on a few droplets the Stokeslet and correction sums cancel as
  well (|V_i| ~ 1e-2 mean |V|), so the reference's per-droplet metric, whose
  floor is 0.01 mean |V|, is held to 1e-4 there;
* Morton tree: theta = 0 equals the corrected direct sum to FP32 accuracy;
  theta = 0.5 keeps the accuracy of the uncorrected walk."""

from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from gpu_util import ETA_OIL, consts, lognormal_state, ref_metric, rel_norm

pytestmark = pytest.mark.gpu


def _corr(g):
    from dem.periodic_correction import COMSOLLatticeCorrection

    return COMSOLLatticeCorrection.from_grid(g["grid_u"], g["grid_v"], g["grid_w"], float(g["L_comsol"]),
                                             float(g["Fz_comsol"]), float(g["eta_comsol"]))


MIXED_V_NORM_TOL = 1e-5
MIXED_V_ABS_TOL = 1e-5  # per droplet, of the mean |V|
MIXED_V_REF_METRIC_TOL = 1e-4


def _check_mixed(V, V_ref):
    assert rel_norm(V, V_ref) <= MIXED_V_NORM_TOL
    err = np.linalg.norm(np.asarray(V) - V_ref, axis=1)
    assert err.max() <= MIXED_V_ABS_TOL * np.linalg.norm(V_ref, axis=1).mean()
    assert ref_metric(V, V_ref)[1] <= MIXED_V_REF_METRIC_TOL


def _direct(n, L, periodic, g, precision="fp64", eta_oil=ETA_OIL):
    from dem.force_calculator import DirectDropletForceCalculator

    fc = DirectDropletForceCalculator(num_particles=n, eps_oil=2.85, eta_oil=eta_oil, eta_water=0.001, E=3e5, L=L,
                                      boundary_mode="periodic" if periodic else "open",
                                      correction_grid_resolution=int(g["grid_resolution"]), precision=precision)
    fc.load_periodic_correction(_corr(g), L_sim=L)
    return fc


@pytest.mark.parametrize("name", ["corr_direct_comsol_periodic_n64.npz", "corr_direct_synth_periodic_n64.npz",
                                  "corr_direct_synth_open_n40.npz"])
def test_fp64_direct_bit_exact_with_reference(golden, name):
    g = golden(name)
    fc = _direct(len(g["radii"]), float(g["L"]), bool(g["periodic"]), g, eta_oil=float(g["eta_oil"]))
    assert fc.corr_enabled[None] == 1 and fc.corr_self_coeff[None] == g["corr_self_coeff"]
    F, V = fc.calculate_forces_and_convection(g["positions"], g["radii"])
    np.testing.assert_array_equal(F, g["forces"])
    np.testing.assert_array_equal(V, g["velocities"])
    V2 = fc.calculate_convection(g["positions"], g["radii"], F)
    np.testing.assert_array_equal(V2, g["velocities"])
    assert fc._ctx.device_errors() == 0


@pytest.mark.parametrize("case", ["corr_direct_comsol_periodic_n64.npz", "corr_direct_synth_open_n40.npz"])
def test_fp64_and_mixed_against_oracle(golden, case):
    g = golden(case)
    periodic = bool(g["periodic"])
    n = 3000
    pos, r, L = lognormal_state(n, seed=41, periodic=periodic)
    m, eta, _ = consts()
    corr = O.Correction(g["grid_u"], g["grid_v"], g["grid_w"], g["grid_min"], g["grid_dx"], g["Fz_comsol"],
                        g["L_comsol"], g["eta_comsol"], L, ETA_OIL, _self_coeff(g, L))
    F_ref = O.direct_forces(pos, r, m, L, periodic)
    V_ref = O.direct_convection_corr(pos, F_ref, eta, L, periodic, corr)
    F, V = _direct(n, L, periodic, g).calculate_forces_and_convection(pos, r)
    np.testing.assert_array_equal(F, F_ref)
    np.testing.assert_array_equal(V, V_ref)
    Fm, Vm = _direct(n, L, periodic, g, precision="mixed").calculate_forces_and_convection(pos, r)
    V_refm = O.direct_convection_corr(pos, Fm, eta, L, periodic, corr)  # the same forces in
    _check_mixed(Vm, V_refm)


def _self_coeff(g, L):
    c = _corr(g)
    d = c.get_grid_data()
    L_ratio = d["L_comsol"] / L
    eta_ratio = d["eta_comsol"] / ETA_OIL
    return float(c.evaluate(np.zeros((1, 3)))[0, 2]) / d["Fz_comsol"] * eta_ratio * L_ratio


def test_mixed_at_65536_against_oracle_rows(golden):
    """The measured size: the FP32 correction pass against the oracle on a
    block of rows (the full oracle sum at this size takes minutes)."""
    g = golden("corr_direct_comsol_periodic_n64.npz")
    n = 65536
    pos, r, L = lognormal_state(n, seed=0)
    m, eta, _ = consts()
    fc = _direct(n, L, True, g, precision="mixed")
    F, V = fc.calculate_forces_and_convection(pos, r)
    rows = (0, 1024)
    corr = O.Correction(g["grid_u"], g["grid_v"], g["grid_w"], g["grid_min"], g["grid_dx"], g["Fz_comsol"],
                        g["L_comsol"], g["eta_comsol"], L, ETA_OIL, _self_coeff(g, L))
    V_ref = O.direct_convection_corr(pos, F, eta, L, True, corr, rows=rows)[: rows[1]]
    _check_mixed(V[: rows[1]], V_ref)
    assert fc._ctx.device_errors() == 0


@pytest.mark.parametrize("name", ["corr_tree_comsol_periodic_mpl2_t05_n120.npz",
                                  "corr_tree_synth_open_mpl1_t07_n120.npz"])
def test_parity_tree_bit_exact_with_reference(golden, name):
    from dem.octree import FlatOctree, TreeDropletForceCalculator

    g = golden(name)
    n, L, per = len(g["radii"]), float(g["L"]), bool(g["periodic"])
    t = FlatOctree(theta=float(g["theta"]), mpl=int(g["mpl"]), num_particles=n,
                   correction_grid_resolution=int(g["grid_resolution"]))
    t.load_periodic_correction(_corr(g), L, eta_sim=float(g["eta_oil"]))
    assert t.corr_self_coeff[None] == g["corr_self_coeff"]
    t.build(g["positions"], g["radii"], L, per)
    F, V = t.compute_forces_and_stokeslet(float(g["m_const"]), float(g["eta_const"]))
    np.testing.assert_array_equal(F, g["forces"])
    np.testing.assert_array_equal(V, g["velocities"])
    t.build(g["positions"], g["radii"], L, per)
    _, VT = t.compute_forces_and_total_velocity(float(g["m_const"]), float(g["eta_const"]), float(g["stokes_factor"]))
    np.testing.assert_array_equal(VT, g["total_velocities"])
    # the calculator keeps the correction across capacity growth (force_tree.py:103-106)
    tc = TreeDropletForceCalculator(num_particles=16, theta=float(g["theta"]), mpl=int(g["mpl"]), eta_oil=ETA_OIL,
                                    L=L, periodic=per, correction_grid_resolution=int(g["grid_resolution"]))
    tc.load_periodic_correction(_corr(g), L)
    F2, V2 = tc.calculate_forces_and_convection(g["positions"], g["radii"])
    np.testing.assert_array_equal(V2, g["velocities"])


def test_parity_tree_against_oracle_tree(golden):
    from dem.octree import FlatOctree

    g = golden("corr_tree_comsol_periodic_mpl2_t05_n120.npz")
    pos, r, L = lognormal_state(2500, seed=43)
    m, eta, _ = consts()
    t = FlatOctree(theta=0.5, mpl=4, num_particles=2500, correction_grid_resolution=int(g["grid_resolution"]))
    t.load_periodic_correction(_corr(g), L, eta_sim=ETA_OIL)
    t.build(pos, r, L, True)
    F, V = t.compute_forces_and_stokeslet(m, eta)
    ot = O.Tree(2500, 0.5, 4)
    ot.set_correction(O.Correction(g["grid_u"], g["grid_v"], g["grid_w"], g["grid_min"], g["grid_dx"],
                                   g["Fz_comsol"], g["L_comsol"], g["eta_comsol"], L, ETA_OIL, _self_coeff(g, L)))
    ot.build(pos, r, L, True)
    F_ref, V_ref = ot.forces_and_stokeslet(m, eta)
    np.testing.assert_array_equal(F, F_ref)
    np.testing.assert_array_equal(V, V_ref)


def test_morton_tree_with_correction(golden):
    from dem.octree import MortonTreeForceCalculator

    g = golden("corr_direct_comsol_periodic_n64.npz")
    n = 4000
    pos, r, L = lognormal_state(n, seed=44)
    m, eta, sf = consts()
    corr = O.Correction(g["grid_u"], g["grid_v"], g["grid_w"], g["grid_min"], g["grid_dx"], g["Fz_comsol"],
                        g["L_comsol"], g["eta_comsol"], L, ETA_OIL, _self_coeff(g, L))

    def calc(theta):
        tc = MortonTreeForceCalculator(num_particles=n, theta=theta, mpl=16, eta_oil=ETA_OIL, L=L, periodic=True,
                                       correction_grid_resolution=int(g["grid_resolution"]))
        tc.load_periodic_correction(_corr(g), L)
        return tc

    F, V = calc(0.0).calculate_forces_and_convection(pos, r)
    V_ref = O.direct_convection_corr(pos, F, eta, L, True, corr)  # theta = 0: every pair exact
    assert rel_norm(V, V_ref) < 2e-5
    tc = calc(0.5)
    F5, V5 = tc.calculate_forces_and_convection(pos, r)
    V5_ref = O.direct_convection_corr(pos, F5, eta, L, True, corr)
    V5_plain = O.direct_convection(pos, F5, eta, L, True)
    # the correction adds no error of its own beyond the monopole truncation it shares
    plain = MortonTreeForceCalculator(num_particles=n, theta=0.5, mpl=16, eta_oil=ETA_OIL, L=L, periodic=True)
    _, V5p = plain.calculate_forces_and_convection(pos, r)
    assert rel_norm(V5, V5_ref) <= 1.1 * rel_norm(V5p, V5_plain) + 1e-4
    _, U = tc.calculate_forces_and_total_velocity(pos, r, sf)
    # total velocity: no self term (flat_tree.py:1326-1588)
    np.testing.assert_allclose(U, V5 + F5 / (sf * r[:, None]) - _self_coeff(g, L) * F5, rtol=1e-9,
                               atol=1e-9 * np.abs(U).max())
    assert tc._ctx.device_errors() == 0


def test_errors():
    from dem.force_calculator import DirectDropletForceCalculator
    from dem.periodic_correction import COMSOLLatticeCorrection

    c = COMSOLLatticeCorrection.from_grid(*(np.zeros((4, 4, 4)),) * 3, L_comsol=1e-3, Fz_comsol=1.0)
    with pytest.raises(RuntimeError):
        DirectDropletForceCalculator(num_particles=8).load_periodic_correction(c, 1e-3)
    with pytest.raises(ValueError):  # grid resolution other than the allocated one
        DirectDropletForceCalculator(num_particles=8, correction_grid_resolution=5).load_periodic_correction(c, 1e-3)
