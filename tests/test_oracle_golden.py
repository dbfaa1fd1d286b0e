"""The CPU oracle against golden vectors produced by the reference's own
``dem/`` classes (tests/golden/make_golden.py).  Bit-exact: the oracle
restates each reference expression in the same order."""

from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN

DIRECT = sorted(p.name for p in GOLDEN.glob("direct_*.npz"))
HASH = sorted(p.name for p in GOLDEN.glob("hash_*.npz"))
MERGE = sorted(p.name for p in GOLDEN.glob("merge_*.npz"))
TREE = sorted(p.name for p in GOLDEN.glob("tree_*.npz"))


@pytest.mark.parametrize("name", DIRECT)
def test_direct_forces_and_convection_bit_exact(golden, name):
    g = golden(name)
    F = O.direct_forces(g["positions"], g["radii"], float(g["m_const"]), float(g["L"]), int(g["periodic"]))
    V = O.direct_convection(g["positions"], F, float(g["eta_const"]), float(g["L"]), int(g["periodic"]))
    np.testing.assert_array_equal(F, g["forces"])
    np.testing.assert_array_equal(V, g["velocities"])


def test_direct_row_ranges_match_full(golden):
    g = golden("direct_periodic_n96.npz")
    args = (float(g["m_const"]), float(g["L"]), int(g["periodic"]))
    full = O.direct_forces(g["positions"], g["radii"], *args)
    part = O.direct_forces(g["positions"], g["radii"], *args, rows=(10, 40))
    np.testing.assert_array_equal(part[10:40], full[10:40])
    assert not part[:10].any() and not part[40:].any()


@pytest.mark.parametrize("name", HASH)
def test_hash_pairs_bit_exact(golden, name):
    g = golden(name)
    hit, pairs = O.hash_detect(g["positions"], g["radii"], float(g["L"]), int(g["periodic"]), table_size=int(g["table_size"]))
    assert hit == bool(g["is_collision"])
    np.testing.assert_array_equal(pairs, g["pairs"])


@pytest.mark.parametrize("name", MERGE)
def test_merge_bit_exact(golden, name):
    g = golden(name)
    p, r, _ = O.merge(g["positions"], g["radii"], g["pairs"])
    np.testing.assert_array_equal(p, g["new_positions"])
    np.testing.assert_array_equal(r, g["new_radii"])


@pytest.mark.parametrize("name", TREE)
def test_tree_bit_exact(golden, name):
    g = golden(name)
    t = O.Tree(len(g["radii"]), float(g["theta"]), int(g["mpl"]))
    t.build(g["positions"], g["radii"], float(g["L"]), bool(g["periodic"]))
    st = t.stats()
    assert st["node_count"] == int(g["node_count"])
    assert st["parent_count"] == int(g["parent_count"])
    assert st["leaf_slot_count"] == int(g["leaf_slot_count"])
    np.testing.assert_array_equal(t.nodes()["count"], g["node_counts"])
    F, V = t.forces_and_stokeslet(float(g["m_const"]), float(g["eta_const"]))
    np.testing.assert_array_equal(F, g["forces"])
    np.testing.assert_array_equal(V, g["velocities"])
    t.build(g["positions"], g["radii"], float(g["L"]), bool(g["periodic"]))
    F2, VT = t.forces_and_total_velocity(float(g["m_const"]), float(g["eta_const"]), float(g["stokes_factor"]))
    np.testing.assert_array_equal(VT, g["total_velocities"])


def test_solver_chain_bit_exact(golden):
    g = golden("solver_direct_periodic_n48.npz")
    chain = O.run_direct_solver(
        g["positions"], g["radii"], float(g["L"]), True, float(g["dt"]), float(g["total_time"]),
        eps_oil=float(g["eps_oil"]), eta_oil=float(g["eta_oil"]), eta_water=float(g["eta_water"]), E=float(g["E"]),
    )
    assert len(chain) == int(g["n_solutions"])
    for k, s in enumerate(chain):
        np.testing.assert_array_equal(s["radii"], g[f"sol{k}_radii"])
        np.testing.assert_array_equal(s["times"], g[f"sol{k}_times"])
        np.testing.assert_array_equal(s["trajectories"], g[f"sol{k}_trajectories"])
        np.testing.assert_array_equal(s["collided"], g[f"sol{k}_collided"])


@pytest.mark.parametrize("n,expected", [(1, 1), (2, 2), (3, 4), (5, 8), (16, 16), (17, 32)])
def test_next_power_of_2(n, expected):
    # spatial_hash_collision_detector.py:18-23 (tests/collision_detector/...:23-25 upstream)
    assert O.next_power_of_2(n) == expected


def test_physics_constants_match_reference_eps0():
    m, eta, sf = O.physics_constants(eps_oil=2.85, eta_oil=0.06, eta_water=0.001, E=3e5)
    assert m == 12 * np.pi * 8.85418781762039e-12 * 2.85 * 3e5**2
    assert abs(m - 85.6184) < 1e-3
    assert abs(eta - 0.66315) < 1e-4
    assert abs(sf - 0.76016) < 1e-4


CORR_DIRECT = sorted(p.name for p in GOLDEN.glob("corr_direct_*.npz"))
CORR_TREE = sorted(p.name for p in GOLDEN.glob("corr_tree_*.npz"))


@pytest.mark.parametrize("name", CORR_DIRECT)
def test_direct_convection_with_correction_bit_exact(golden, name):
    g = golden(name)
    c = O.Correction.from_golden(g)
    assert (c.Fz_inv, c.cL, c.eta_r) == (float(g["corr_Fz_inv"]), float(g["corr_L_ratio"]), float(g["corr_eta_ratio"]))
    L, per = float(g["L"]), int(g["periodic"])
    F = O.direct_forces(g["positions"], g["radii"], float(g["m_const"]), L, per)
    V = O.direct_convection_corr(g["positions"], F, float(g["eta_const"]), L, per, c)
    np.testing.assert_array_equal(F, g["forces"])
    np.testing.assert_array_equal(V, g["velocities"])
    # the correction is not negligible in these cases
    V0 = O.direct_convection(g["positions"], F, float(g["eta_const"]), L, per)
    assert np.linalg.norm(V - V0) > 1e-3 * np.linalg.norm(V)


@pytest.mark.parametrize("name", CORR_TREE)
def test_tree_velocity_with_correction_bit_exact(golden, name):
    g = golden(name)
    t = O.Tree(len(g["radii"]), float(g["theta"]), int(g["mpl"]))
    t.set_correction(O.Correction.from_golden(g))
    args = (g["positions"], g["radii"], float(g["L"]), bool(g["periodic"]))
    t.build(*args)
    F, V = t.forces_and_stokeslet(float(g["m_const"]), float(g["eta_const"]))
    t.build(*args)
    _, VT = t.forces_and_total_velocity(float(g["m_const"]), float(g["eta_const"]), float(g["stokes_factor"]))
    np.testing.assert_array_equal(F, g["forces"])
    np.testing.assert_array_equal(V, g["velocities"])
    np.testing.assert_array_equal(VT, g["total_velocities"])
