"""Periodic-image correction of the Stokeslet from a COMSOL solution.

Drop-in for dem/periodic_correction/comsol_lattice_correction.py:8-328 of
ddkx21/particle-simulator.  COMSOL solved the flow of one droplet pulled by a
z-force in a periodic cell and subtracted the free-space Stokeslet; what is
left (u2, v2, w2 in ``U_lattice.txt``) is the velocity of the periodic images.
The data cover the quarter cell [0, L/2]^2 x [-L/2, L/2].  This class

* mirrors them to the full cell with the parities of a z-Stokeslet (u odd in
  x, even in y; v even in x, odd in y; w even in both), :107-168;
* resamples them on a regular n^3 grid over [-L/2, L/2]^3 (piecewise-linear
  interpolation on the Delaunay triangulation, nearest data point where that
  is undefined), :170-220;
* evaluates the correction of an arbitrary force direction from the three
  permuted lookups of the z-column, :246-296;
* hands the grid to the calculators (``get_grid_data``), :298-328.

This is one-time host preprocessing (scipy); the per-pair lookups run in the
CUDA kernels of libdem_b200 once a calculator's ``load_periodic_correction``
has uploaded the grid.
"""

from __future__ import annotations

import json
import os
from pathlib import Path

import numpy as np

DATA_ENV = "DEM_COMSOL_DATA"


class COMSOLLatticeCorrection:
    @classmethod
    def load_default(cls):
        """The shipped COMSOL solution (comsol_lattice_correction.py:25-28).

        The data are not redistributed with this package: the directory is
        taken from the ``DEM_COMSOL_DATA`` environment variable, else a
        ``data`` directory next to this module.  Point it at the reference's
        ``dem/periodic_correction/data`` (``U_lattice.txt`` +
        ``comsol_params.json``)."""
        env = os.environ.get(DATA_ENV)
        d = Path(env) if env else Path(__file__).resolve().parent / "data"
        if not (d / "comsol_params.json").exists():
            raise FileNotFoundError(
                f"COMSOL correction data not found in {d}: set {DATA_ENV} to a directory holding "
                "comsol_params.json and its velocity file, or use from_data_dir()")
        return cls.from_data_dir(str(d))

    @classmethod
    def from_data_dir(cls, data_dir: str):
        """comsol_lattice_correction.py:30-58: every parameter from comsol_params.json."""
        params = json.loads((Path(data_dir) / "comsol_params.json").read_text())
        R, E0 = params["R"], params["E0"]
        Fz_comsol = 4 * np.pi * R**2 * params["eps_0"] * params["eps_r"] * E0**2  # force on the COMSOL drop
        return cls(
            data_path=os.path.join(data_dir, params["velocity_file"]),
            L_comsol=params["L"],
            Fz_comsol=Fz_comsol,
            eta_comsol=params["eta"],
            grid_resolution=params.get("grid_resolution", 48),
        )

    @classmethod
    def from_grid(cls, grid_u, grid_v, grid_w, L_comsol: float, Fz_comsol: float, eta_comsol: float = 0.065):
        """A correction given directly on the regular grid linspace(-L/2, L/2, n)
        per axis (no COMSOL file): (n, n, n) arrays indexed [ix, iy, iz]."""
        grids = [np.array(g, dtype=np.float64) for g in (grid_u, grid_v, grid_w)]
        n = grids[0].shape[0]
        if n < 2 or any(g.shape != (n, n, n) for g in grids):
            raise ValueError("grids must be three (n, n, n) arrays with n >= 2")
        self = cls.__new__(cls)
        self.L_comsol, self.Fz_comsol, self.eta_comsol, self.grid_resolution = L_comsol, Fz_comsol, eta_comsol, n
        self.grid_coords = np.linspace(-L_comsol / 2.0, L_comsol / 2.0, n)
        self.grid_u, self.grid_v, self.grid_w = grids
        self._interp = self._regular_interpolators()
        return self

    def __init__(self, data_path: str, L_comsol: float, Fz_comsol: float, eta_comsol: float = 0.065,
                 grid_resolution: int = 48):
        self.L_comsol = L_comsol
        self.Fz_comsol = Fz_comsol
        self.eta_comsol = eta_comsol
        self.grid_resolution = grid_resolution
        points, uvw = self._read(data_path)
        points, uvw = self._mirror(points, uvw)
        self.grid_coords, (self.grid_u, self.grid_v, self.grid_w) = self._resample(points, uvw, grid_resolution)
        self._interp = self._regular_interpolators()

    # -- preprocessing ---------------------------------------------------------
    @staticmethod
    def _read(data_path):
        """Columns x y z u2 v2 w2 (p2 ignored); '%' starts a comment (:94-105)."""
        data = np.loadtxt(data_path, comments="%")
        points, uvw = data[:, 0:3], data[:, 3:6]
        if np.any(points[:, 0] < -1e-15) or np.any(points[:, 1] < -1e-15):
            raise ValueError("the COMSOL data must cover the quarter cell x >= 0, y >= 0")
        return points, uvw

    @staticmethod
    def _mirror(points, uvw):
        """Quarter cell -> full cell.  Reflections x -> -x (points with x > 0),
        y -> -y (y > 0) and both (x > 0 and y > 0) are appended in that order;
        the sign pattern per component is that of a z-Stokeslet."""
        eps = 1e-15  # points on the symmetry planes are not duplicated
        px, py = points[:, 0] > eps, points[:, 1] > eps
        parts_p, parts_v = [points], [uvw]
        for mask, flip, sign in ((px, (-1.0, 1.0, 1.0), (-1.0, 1.0, 1.0)),
                                 (py, (1.0, -1.0, 1.0), (1.0, -1.0, 1.0)),
                                 (px & py, (-1.0, -1.0, 1.0), (-1.0, -1.0, 1.0))):
            if np.any(mask):
                parts_p.append(points[mask] * np.array(flip))
                parts_v.append(uvw[mask] * np.array(sign))
        return np.concatenate(parts_p), np.concatenate(parts_v)

    def _resample(self, points, uvw, n):
        from scipy.interpolate import LinearNDInterpolator, NearestNDInterpolator
        from scipy.spatial import Delaunay

        half = self.L_comsol / 2.0
        axis = np.linspace(-half, half, n)
        g = np.meshgrid(axis, axis, axis, indexing="ij")
        query = np.column_stack([c.ravel() for c in g])
        # one triangulation and one point location for the three components
        vals = LinearNDInterpolator(Delaunay(points), uvw)(query)
        bad = np.isnan(vals)
        if np.any(bad):  # outside the convex hull: nearest data point
            rows = np.any(bad, axis=1)
            near = NearestNDInterpolator(points, uvw)(query[rows])
            vals[rows] = np.where(bad[rows], near, vals[rows])
        return axis, [np.ascontiguousarray(vals[:, k]).reshape(n, n, n) for k in range(3)]

    def _regular_interpolators(self):
        from scipy.interpolate import RegularGridInterpolator

        c = self.grid_coords
        return tuple(RegularGridInterpolator((c, c, c), g, method="linear", bounds_error=False, fill_value=0.0)
                     for g in (self.grid_u, self.grid_v, self.grid_w))

    # -- evaluation ------------------------------------------------------------
    def evaluate(self, r_rel: np.ndarray, F_j: np.ndarray = None) -> np.ndarray:
        """Correction velocity at offsets r_rel (M, 3) in COMSOL coordinates
        (zero outside the grid).  Without F_j: the raw z-column (u, v, w); with
        F_j (M, 3): the full tensor contracted with F_j / Fz_comsol, using the
        cubic symmetry of the lattice, G_x(x,y,z) = (w, v, u)(z, y, x) and
        G_y(x,y,z) = (u, w, v)(x, z, y)."""
        iu, iv, iw = self._interp
        r_rel = np.asarray(r_rel, dtype=np.float64)
        if F_j is None:
            return np.column_stack([iu(r_rel), iv(r_rel), iw(r_rel)])
        Fz_inv = 1.0 / self.Fz_comsol
        pz, px, py = r_rel, r_rel[:, [2, 1, 0]], r_rel[:, [0, 2, 1]]
        gz = (iu(pz), iv(pz), iw(pz))
        gx = (iw(px), iv(px), iu(px))
        gy = (iu(py), iw(py), iv(py))
        F_j = np.asarray(F_j, dtype=np.float64)
        sx, sy, sz = F_j[:, 0] * Fz_inv, F_j[:, 1] * Fz_inv, F_j[:, 2] * Fz_inv
        return np.column_stack([gx[k] * sx + gy[k] * sy + gz[k] * sz for k in range(3)])

    def get_grid_data(self) -> dict:
        """The regular grid and the COMSOL run's parameters (:298-328)."""
        return {
            "grid_u": self.grid_u.copy(),
            "grid_v": self.grid_v.copy(),
            "grid_w": self.grid_w.copy(),
            "grid_min": self.grid_coords[0],
            "grid_max": self.grid_coords[-1],
            "grid_dx": self.grid_coords[1] - self.grid_coords[0],
            "grid_resolution": self.grid_resolution,
            "L_comsol": self.L_comsol,
            "Fz_comsol": self.Fz_comsol,
            "eta_comsol": self.eta_comsol,
        }


def to_device(ctx, correction, L_sim: float, eta_sim: float | None, resolution: int):
    """What load_periodic_correction does with a correction object
    (direct_droplet_force_calculator.py:74-120, flat_tree.py:141-167): the
    scale factors

        L_ratio = L_comsol / L_sim,  eta_ratio = eta_comsol / eta_sim (1 without eta_sim),
        self_coeff = w(0,0,0) / Fz_comsol * eta_ratio * L_ratio   (w from correction.evaluate)

    and the grid uploaded to ``ctx``'s device.  Returns (device grid, scalars)."""
    from .. import _native as N

    grid_data = correction.get_grid_data()
    n = int(grid_data["grid_resolution"])
    if n != int(resolution):
        raise ValueError(f"the correction grid is {n}^3 but the calculator was created with "
                         f"correction_grid_resolution={resolution}")
    L_ratio = grid_data["L_comsol"] / L_sim
    eta_ratio = grid_data["eta_comsol"] / eta_sim if eta_sim is not None else 1.0
    w_self = float(correction.evaluate(np.array([[0.0, 0.0, 0.0]]))[0, 2])
    self_coeff = w_self / grid_data["Fz_comsol"] * eta_ratio * L_ratio
    scalars = dict(grid_min=grid_data["grid_min"], inv_dx=1.0 / grid_data["grid_dx"], n=n,
                   Fz_inv=1.0 / grid_data["Fz_comsol"], L_ratio=L_ratio, eta_ratio=eta_ratio, self_coeff=self_coeff)
    dev = N.Correction(ctx, grid_data["grid_u"], grid_data["grid_v"], grid_data["grid_w"], scalars["grid_min"],
                       scalars["inv_dx"], scalars["Fz_inv"], L_ratio, eta_ratio, self_coeff)
    return dev, scalars


class ScalarField:
    """``f[None]`` read access to a value, like a 0-d Taichi field."""

    __slots__ = ("value",)

    def __init__(self, value=0):
        self.value = value

    def __getitem__(self, key):
        return self.value


def correction_fields(scalars: dict | None) -> dict:
    """The reference calculators' corr_* scalar fields for the given scalars
    (None: correction off, as before load_periodic_correction)."""
    s = scalars or {}
    return {
        "corr_enabled": ScalarField(1 if scalars else 0),
        "corr_grid_min": ScalarField(s.get("grid_min", 0.0)),
        "corr_grid_inv_dx": ScalarField(s.get("inv_dx", 0.0)),
        "corr_grid_n": ScalarField(s.get("n", 0)),
        "corr_Fz_inv": ScalarField(s.get("Fz_inv", 0.0)),
        "corr_L_ratio": ScalarField(s.get("L_ratio", 0.0)),
        "corr_eta_ratio": ScalarField(s.get("eta_ratio", 0.0)),
        "corr_self_coeff": ScalarField(s.get("self_coeff", 0.0)),
    }
