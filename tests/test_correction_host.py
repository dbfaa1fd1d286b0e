"""Host side of the periodic-image correction: COMSOLLatticeCorrection against
the reference's own loader output (tests/golden/corr_grid_comsol_r12.npz, made
by tests/golden/make_golden.py from the reference's class and its shipped
data), the reference's own checks of that class
(tests/periodic_correction/test_comsol_lattice_correction.py), and the
scalars load_periodic_correction derives."""

from __future__ import annotations

import os
from pathlib import Path

import numpy as np
import pytest

from dem.periodic_correction import COMSOLLatticeCorrection
from dem.periodic_correction.comsol_lattice_correction import DATA_ENV

# the reference checkout, named by DEM_REFERENCE (as for tests/golden/make_golden.py); the
# test that reads its COMSOL data is skipped when the variable is unset
_REF = os.environ.get("DEM_REFERENCE")
REF_DATA = Path(_REF) / "dem" / "periodic_correction" / "data" if _REF else None


@pytest.fixture(scope="module")
def grid12(golden):
    g = golden("corr_grid_comsol_r12.npz")
    c = COMSOLLatticeCorrection.from_grid(g["grid_u"], g["grid_v"], g["grid_w"], float(g["L_comsol"]),
                                          float(g["Fz_comsol"]), float(g["eta_comsol"]))
    return g, c


def test_evaluate_matches_reference(grid12):
    g, c = grid12
    np.testing.assert_array_equal(c.evaluate(g["probe"]), g["eval_raw"])
    np.testing.assert_array_equal(c.evaluate(g["probe"], g["probe_F"]), g["eval_F"])
    np.testing.assert_array_equal(c.evaluate(np.zeros((1, 3))), g["eval_origin"])


def test_grid_data(grid12):
    g, c = grid12
    d = c.get_grid_data()
    for key in ("grid_u", "grid_v", "grid_w", "grid_min", "grid_max", "grid_dx", "grid_resolution", "L_comsol",
                "Fz_comsol", "eta_comsol"):
        assert key in d
    assert d["grid_min"] == g["grid_min"] and d["grid_dx"] == g["grid_dx"] and d["grid_max"] == g["grid_max"]
    np.testing.assert_allclose(d["grid_min"], -d["grid_max"])
    n = d["grid_resolution"]
    np.testing.assert_allclose(d["grid_dx"], (d["grid_max"] - d["grid_min"]) / (n - 1), rtol=1e-12)
    assert d["grid_u"].shape == (n, n, n) and not np.any(np.isnan(d["grid_w"]))


def test_reference_checks_of_evaluate(grid12):
    _, c = grid12
    L = c.L_comsol
    r = np.array([[L * 0.1, 0.0, 0.0]])
    np.testing.assert_allclose(c.evaluate(r, np.array([[0.0, 0.0, c.Fz_comsol]])), c.evaluate(r), atol=1e-12)
    far = L * 10
    np.testing.assert_array_equal(c.evaluate(np.array([[far, far, far]])), np.zeros((1, 3)))
    x = L * 0.15  # mirror parities of the z-Stokeslet correction
    np.testing.assert_allclose(c.evaluate([[x, 0, 0]])[0, 0], -c.evaluate([[-x, 0, 0]])[0, 0], atol=1e-10)
    np.testing.assert_allclose(c.evaluate([[0, x, 0]])[0, 1], -c.evaluate([[0, -x, 0]])[0, 1], atol=1e-10)
    np.testing.assert_allclose(c.evaluate([[x, x, 0]])[0, 2], c.evaluate([[-x, -x, 0]])[0, 2], atol=1e-10)


def test_from_grid_rejects_bad_shapes():
    with pytest.raises(ValueError):
        COMSOLLatticeCorrection.from_grid(np.zeros((3, 3, 3)), np.zeros((3, 3, 3)), np.zeros((3, 3, 2)), 1e-3, 1.0)
    with pytest.raises(ValueError):
        COMSOLLatticeCorrection.from_grid(np.zeros((1, 1, 1)), np.zeros((1, 1, 1)), np.zeros((1, 1, 1)), 1e-3, 1.0)


def test_load_default_needs_the_data(monkeypatch, tmp_path):
    monkeypatch.setenv(DATA_ENV, str(tmp_path))
    with pytest.raises(FileNotFoundError):
        COMSOLLatticeCorrection.load_default()


@pytest.mark.skipif(REF_DATA is None or not REF_DATA.exists(),
                    reason="DEM_REFERENCE does not name a reference checkout with its COMSOL data")
def test_loader_reproduces_reference_grid(golden, monkeypatch):
    g = golden("corr_grid_comsol_r12.npz")
    import json

    prm = json.loads((REF_DATA / "comsol_params.json").read_text())
    c = COMSOLLatticeCorrection(data_path=str(REF_DATA / prm["velocity_file"]), L_comsol=prm["L"],
                                Fz_comsol=float(g["Fz_comsol"]), eta_comsol=prm["eta"], grid_resolution=12)
    d = c.get_grid_data()
    for k in ("grid_u", "grid_v", "grid_w", "grid_min", "grid_dx"):
        np.testing.assert_array_equal(d[k], g[k])
    monkeypatch.setenv(DATA_ENV, str(REF_DATA))
    c48 = COMSOLLatticeCorrection.load_default()
    assert c48.grid_resolution == 48 and c48.Fz_comsol == g["Fz_comsol"]


def test_scalars_follow_load_periodic_correction(golden, grid12):
    """The scale factors and the self coefficient, computed as the reference's
    load_periodic_correction does, equal the reference's own values."""
    from dem.periodic_correction.comsol_lattice_correction import correction_fields

    for name in ("corr_direct_comsol_periodic_n64.npz", "corr_direct_synth_open_n40.npz"):
        g = golden(name)
        c = COMSOLLatticeCorrection.from_grid(g["grid_u"], g["grid_v"], g["grid_w"], float(g["L_comsol"]),
                                              float(g["Fz_comsol"]), float(g["eta_comsol"]))
        d = c.get_grid_data()
        L_ratio = d["L_comsol"] / float(g["L"])
        eta_ratio = d["eta_comsol"] / float(g["eta_oil"])
        w_self = float(c.evaluate(np.array([[0.0, 0.0, 0.0]]))[0, 2])
        assert L_ratio == g["corr_L_ratio"] and eta_ratio == g["corr_eta_ratio"]
        assert w_self / d["Fz_comsol"] * eta_ratio * L_ratio == g["corr_self_coeff"]
        f = correction_fields(dict(self_coeff=1.5))
        assert f["corr_enabled"][None] == 1 and f["corr_self_coeff"][None] == 1.5
        assert correction_fields(None)["corr_enabled"][None] == 0
