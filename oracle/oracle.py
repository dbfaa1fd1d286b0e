"""ctypes front-end of the CPU oracle (``oracle/dem_oracle.c``).

TEST INFRASTRUCTURE ONLY: the checker that the CUDA product is compared
against, and the CPU baseline timed by ``bench.py``.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs import this module.

Each function restates one reference function (file:line of
ddkx21/particle-simulator given in the docstring) with numpy-compatible
inputs: positions ``(N, 3)`` float64, radii ``(N,)`` float64.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

EPS0 = 8.85418781762039e-12  # direct_droplet_force_calculator.py:23


def build(force: bool = False) -> Path:
    """Compile ``liboracle.so`` with the recipe in ``oracle/Makefile``."""
    if force or not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < (HERE / "dem_oracle.c").stat().st_mtime:
        env = dict(os.environ)
        env.pop("CC", None)
        subprocess.run(["make", "-s", "-C", str(HERE), "-B" if force else "liboracle.so"], check=True, env=env)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB_PATH))
        d, i, i64, vp = C.c_double, C.c_int, C.c_int64, C.c_void_p
        P = C.POINTER
        pd, pi32, pi64 = P(C.c_double), P(C.c_int32), P(C.c_int64)
        L.dem_oracle_max_threads.restype = i
        L.dem_oracle_direct_forces.argtypes = [i, pd, pd, pd, pd, d, d, i, pd, pd, pd, i, i, i]
        L.dem_oracle_direct_convection.argtypes = [i, pd, pd, pd, pd, pd, pd, d, d, i, pd, pd, pd, i, i, i]
        L.dem_oracle_direct_convection_corr.argtypes = [i, pd, pd, pd, pd, pd, pd, d, d, i, i, pd, pd, pd, d, d, d,
                                                        d, d, d, pd, pd, pd, i, i, i]
        L.dem_oracle_tree_set_correction.argtypes = [vp, i, pd, pd, pd, d, d, d, d, d, d]
        L.dem_oracle_euler_direct.argtypes = [i, pd, pd, pd, pd, d, d, d, i]
        L.dem_oracle_euler_total.argtypes = [i, pd, pd, d, d, i]
        L.dem_oracle_hash_detect.argtypes = [i, pd, pd, d, i, i, pi32, i64, pi64]
        L.dem_oracle_hash_detect.restype = i64
        L.dem_oracle_merge.argtypes = [i, pd, pd, pi32, i, pd, pd, pi32]
        L.dem_oracle_merge.restype = i
        L.dem_oracle_tree_create.argtypes = [i, i, d, i]
        L.dem_oracle_tree_create.restype = vp
        L.dem_oracle_tree_destroy.argtypes = [vp]
        L.dem_oracle_tree_set_params.argtypes = [vp, d, i]
        L.dem_oracle_tree_build.argtypes = [vp, i, pd, pd, d, i]
        L.dem_oracle_tree_build.restype = i
        L.dem_oracle_tree_forces.argtypes = [vp, d, pd, i, i, i]
        L.dem_oracle_tree_propagate_forces.argtypes = [vp, pd]
        L.dem_oracle_tree_velocity.argtypes = [vp, pd, d, d, pd, i, i, i]
        L.dem_oracle_tree_stats.argtypes = [vp, pi64]
        L.dem_oracle_tree_nodes.argtypes = [vp, pi32, pi32, pi32, pi32, pd, pd]
        L.dem_oracle_tree_leaf_indices.argtypes = [vp, pi32]
        _lib = L
    return _lib


def _pd(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _pi(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def max_threads() -> int:
    return int(lib().dem_oracle_max_threads())


def physics_constants(eps_oil=2.85, eta_oil=0.065, eta_water=0.001, E=3e5):
    """m_const, eta_const (direct_droplet_force_calculator.py:30-31) and the
    Hadamard-Rybczynski stokes factor (euler_droplet_solver.py:39-41)."""
    m_const = 12 * np.pi * EPS0 * eps_oil * E**2
    eta_const = 1 / (8 * np.pi * eta_oil)
    stokes = 2 * np.pi * eta_oil * (2 * eta_oil + 3 * eta_water) / (eta_oil + eta_water)
    return m_const, eta_const, stokes


def _rows(n, rows):
    if rows is None:
        return 0, n
    return int(rows[0]), int(rows[1])


def direct_forces(pos, r, m_const, L, periodic, rows=None, threads=0):
    """_calculate_forces, direct_droplet_force_calculator.py:202-253."""
    pos = _f64(pos).reshape(-1, 3)
    r = _f64(r)
    n = len(r)
    x, y, z = (_f64(pos[:, k]) for k in range(3))
    out = np.zeros((3, n))
    i0, i1 = _rows(n, rows)
    lib().dem_oracle_direct_forces(
        n, _pd(x), _pd(y), _pd(z), _pd(r), m_const, L, int(periodic), _pd(out[0]), _pd(out[1]), _pd(out[2]), i0, i1, threads
    )
    return np.ascontiguousarray(out.T)


def direct_convection(pos, F, eta_const, L, periodic, rows=None, threads=0):
    """_calculate_convection_velocities, direct_droplet_force_calculator.py:354-468
    (periodic correction off)."""
    pos = _f64(pos).reshape(-1, 3)
    F = _f64(F).reshape(-1, 3)
    n = len(pos)
    x, y, z = (_f64(pos[:, k]) for k in range(3))
    fx, fy, fz = (_f64(F[:, k]) for k in range(3))
    out = np.zeros((3, n))
    i0, i1 = _rows(n, rows)
    lib().dem_oracle_direct_convection(
        n, _pd(x), _pd(y), _pd(z), _pd(fx), _pd(fy), _pd(fz), eta_const, L, int(periodic),
        _pd(out[0]), _pd(out[1]), _pd(out[2]), i0, i1, threads,
    )
    return np.ascontiguousarray(out.T)


class Correction:
    """Parameters of the periodic-image Oseen correction as the reference loads
    them (direct_droplet_force_calculator.py:74-120, flat_tree.py:141-167):
    the regular n^3 grids and

        ginv = 1 / grid_dx,  Fz_inv = 1 / Fz_comsol,  cL = L_comsol / L_sim,
        eta_r = eta_comsol / eta_sim,  g_self = w(0,0,0) / Fz_comsol * eta_r * cL.
    """

    def __init__(self, grid_u, grid_v, grid_w, grid_min, grid_dx, Fz_comsol, L_comsol, eta_comsol, L_sim, eta_sim,
                 self_coeff):
        self.u, self.v, self.w = (np.ascontiguousarray(g, dtype=np.float64) for g in (grid_u, grid_v, grid_w))
        self.n = int(self.u.shape[0])
        self.gmin = float(grid_min)
        self.ginv = 1.0 / float(grid_dx)
        self.Fz_inv = 1.0 / float(Fz_comsol)
        self.cL = float(L_comsol) / float(L_sim)
        self.eta_r = float(eta_comsol) / float(eta_sim)
        self.g_self = float(self_coeff)

    @classmethod
    def from_golden(cls, g):
        """From a tests/golden corr_* case (the grid and the reference's own self coefficient)."""
        return cls(g["grid_u"], g["grid_v"], g["grid_w"], g["grid_min"], g["grid_dx"], g["Fz_comsol"],
                   g["L_comsol"], g["eta_comsol"], g["L"], g["eta_oil"], g["corr_self_coeff"])

    def args(self):
        return (self.n, _pd(self.u), _pd(self.v), _pd(self.w), self.gmin, self.ginv, self.Fz_inv, self.cL,
                self.eta_r, self.g_self)


def direct_convection_corr(pos, F, eta_const, L, periodic, corr: Correction, rows=None, threads=0):
    """_calculate_convection_velocities with the periodic-image correction on,
    direct_droplet_force_calculator.py:354-464."""
    pos = _f64(pos).reshape(-1, 3)
    F = _f64(F).reshape(-1, 3)
    n = len(pos)
    x, y, z = (_f64(pos[:, k]) for k in range(3))
    fx, fy, fz = (_f64(F[:, k]) for k in range(3))
    out = np.zeros((3, n))
    i0, i1 = _rows(n, rows)
    lib().dem_oracle_direct_convection_corr(
        n, _pd(x), _pd(y), _pd(z), _pd(fx), _pd(fy), _pd(fz), eta_const, L, int(periodic), *corr.args(),
        _pd(out[0]), _pd(out[1]), _pd(out[2]), i0, i1, threads,
    )
    return np.ascontiguousarray(out.T)


def euler_direct(pos, r, F, V, stokes_factor, dt, L, periodic):
    """euler_droplet_solver.py:121-131 on a copy of ``pos``."""
    p = _f64(pos).reshape(-1, 3).copy()
    r = _f64(r)
    lib().dem_oracle_euler_direct(len(r), _pd(p), _pd(r), _pd(_f64(F)), _pd(_f64(V)), stokes_factor, dt, L, int(periodic))
    return p


def euler_total(pos, Vt, dt, L, periodic):
    """euler_droplet_solver.py:119, :130-131 on a copy of ``pos``."""
    p = _f64(pos).reshape(-1, 3).copy()
    lib().dem_oracle_euler_total(len(p), _pd(p), _pd(_f64(Vt)), dt, L, int(periodic))
    return p


def next_power_of_2(n: int) -> int:
    """spatial_hash_collision_detector.py:18-23."""
    p = 1
    while p < n:
        p <<= 1
    return p


def hash_detect(pos, r, L, periodic, table_size=None, capacity=None):
    """SpatialHashCollisionDetector.detect, spatial_hash_collision_detector.py:233-316.

    ``table_size`` defaults to next_pow2(2 * capacity) as in ``__init__``
    (:42); ``capacity`` defaults to N.  Returns ``(is_collision, pairs)`` with
    every unique pair (the reference's own pair buffer drops hits beyond its
    capacity, :227-229; the oracle keeps them all)."""
    pos = _f64(pos).reshape(-1, 3)
    r = _f64(r)
    n = len(r)
    if capacity is None:
        capacity = n
    if table_size is None:
        table_size = next_power_of_2(2 * capacity)
    cap = 4 * n + 64
    while True:
        out = np.zeros((cap, 2), dtype=np.int32)
        raw = C.c_int64(0)
        k = lib().dem_oracle_hash_detect(n, _pd(pos), _pd(r), float(L), int(periodic), int(table_size), _pi(out), cap, C.byref(raw))
        if k >= 0:
            break
        cap = -k
    return bool(raw.value > 0), out[:k].copy()


def merge(pos, r, pairs):
    """DropletSolution.generate_next_solution, droplet_solution.py:208-287.

    Pairs are ordered by (i, j) before the greedy pass (the reference orders
    them by column 0, :229-230).  Returns (new_pos, new_r, merged_pairs)."""
    pos = _f64(pos).reshape(-1, 3)
    r = _f64(r)
    pairs = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
    if len(pairs):
        order = np.lexsort((pairs[:, 1], pairs[:, 0]))
        pairs = np.ascontiguousarray(pairs[order])
    n, k = len(r), len(pairs)
    out_p = np.zeros((n, 3))
    out_r = np.zeros(n)
    mp = np.zeros((max(k, 1), 2), dtype=np.int32)
    w = lib().dem_oracle_merge(n, _pd(pos), _pd(r), _pi(pairs), k, _pd(out_p), _pd(out_r), _pi(mp))
    m = n - w
    return out_p[:w].copy(), out_r[:w].copy(), mp[:m].copy()


class Tree:
    """FlatOctree, flat_tree.py:36-1630 (periodic-image correction optional)."""

    def __init__(self, num_particles, theta=0.5, mpl=1, max_nodes=0):
        self.h = lib().dem_oracle_tree_create(int(num_particles), int(mpl), float(theta), int(max_nodes))
        self.theta, self.mpl = theta, mpl

    def __del__(self):
        if getattr(self, "h", None):
            lib().dem_oracle_tree_destroy(self.h)
            self.h = None

    def update_params(self, theta, mpl):
        self.theta, self.mpl = theta, mpl
        lib().dem_oracle_tree_set_params(self.h, float(theta), int(mpl))

    def set_correction(self, corr: Correction | None):
        """load_periodic_correction, flat_tree.py:141-167 (None switches it off)."""
        self._corr = corr  # the C side borrows the grids
        if corr is None:
            lib().dem_oracle_tree_set_correction(self.h, 0, None, None, None, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0)
        else:
            lib().dem_oracle_tree_set_correction(self.h, *corr.args())

    def build(self, pos, r, L, periodic=False):
        pos = _f64(pos).reshape(-1, 3)
        r = _f64(r)
        self.n = len(r)
        if lib().dem_oracle_tree_build(self.h, self.n, _pd(pos), _pd(r), float(L), int(bool(periodic))) != 0:
            raise ValueError("number of particles exceeds the tree capacity")

    def stats(self):
        out = np.zeros(6, dtype=np.int64)
        lib().dem_oracle_tree_stats(self.h, out.ctypes.data_as(C.POINTER(C.c_int64)))
        keys = ("node_count", "parent_count", "leaf_slot_count", "max_nodes", "n_levels", "num_particles")
        return {k: int(v) for k, v in zip(keys, out)}

    def nodes(self):
        nc = self.stats()["node_count"]
        cnt, fc, nx, ls = (np.zeros(nc, dtype=np.int32) for _ in range(4))
        r3 = np.zeros((nc, 4))
        fs = np.zeros((nc, 12))
        lib().dem_oracle_tree_nodes(self.h, _pi(cnt), _pi(fc), _pi(nx), _pi(ls), _pd(r3), _pd(fs))
        return dict(count=cnt, first_child=fc, next=nx, leaf_start=ls, r3=r3, fs=fs)

    def leaf_indices(self):
        out = np.zeros(self.n, dtype=np.int32)
        lib().dem_oracle_tree_leaf_indices(self.h, _pi(out))
        return out

    def forces(self, m_const, rows=None, threads=0):
        """compute_forces, flat_tree.py:896-906."""
        f = np.zeros((self.n, 3))
        i0, i1 = _rows(self.n, rows)
        lib().dem_oracle_tree_forces(self.h, float(m_const), _pd(f), i0, i1, threads)
        return f

    def propagate_forces(self, forces=None):
        lib().dem_oracle_tree_propagate_forces(self.h, None if forces is None else _pd(_f64(forces)))

    def velocity(self, forces, eta_const, stokes_factor=0.0, rows=None, threads=0):
        """_compute_stokeslet_kernel (stokes_factor=0) or
        _compute_total_velocity_kernel (stokes_factor>0)."""
        forces = _f64(forces).reshape(-1, 3)
        v = np.zeros((self.n, 3))
        i0, i1 = _rows(self.n, rows)
        lib().dem_oracle_tree_velocity(self.h, _pd(forces), float(eta_const), float(stokes_factor), _pd(v), i0, i1, threads)
        return v

    def forces_and_stokeslet(self, m_const, eta_const):
        """compute_forces_and_stokeslet, flat_tree.py:1314-1324."""
        f = self.forces(m_const)
        self.propagate_forces()
        return f, self.velocity(f, eta_const)

    def forces_and_total_velocity(self, m_const, eta_const, stokes_factor):
        """compute_forces_and_total_velocity, flat_tree.py:1606-1612."""
        f = self.forces(m_const)
        self.propagate_forces()
        return f, self.velocity(f, eta_const, stokes_factor)


def run_direct_solver(pos, r, L, periodic, dt, total_time, eps_oil=2.85, eta_oil=0.065, eta_water=0.001, E=3e5,
                      capacity=None, t0=0.0):
    """EulerDropletSolver.solve (euler_droplet_solver.py:43-159) with the direct
    calculator and the spatial-hash detector, restated on the oracle kernels.

    Returns the chain of solutions as a list of dicts with ``radii``,
    ``times`` and ``trajectories`` (every step saved) and ``collided``."""
    m_const, eta_const, sf = physics_constants(eps_oil, eta_oil, eta_water, E)
    pos = _f64(pos).reshape(-1, 3).copy()
    r = _f64(r).copy()
    cap = len(r) if capacity is None else capacity
    table = next_power_of_2(2 * cap)
    t = float(t0)
    t_end = t + float(total_time)
    chain = [dict(radii=r.copy(), times=[t], trajectories=[pos.copy()], collided=np.zeros((0, 2), np.int32))]
    while t < t_end:
        remaining = int((t_end - t) / dt) + 1
        merged = False
        for _ in range(remaining):
            hit, pairs = hash_detect(pos, r, L, periodic, table_size=table)
            if hit:
                chain[-1]["collided"] = pairs
                pos, r, _ = merge(pos, r, pairs)
                chain.append(dict(radii=r.copy(), times=[t], trajectories=[pos.copy()], collided=np.zeros((0, 2), np.int32)))
                merged = True
                break
            F = direct_forces(pos, r, m_const, L, periodic)
            V = direct_convection(pos, F, eta_const, L, periodic)
            pos = euler_direct(pos, r, F, V, sf, dt, L, periodic)
            t += dt
            chain[-1]["times"].append(t)
            chain[-1]["trajectories"].append(pos.copy())
        if not merged and t >= t_end:
            break
    for s in chain:
        s["times"] = np.asarray(s["times"])
        s["trajectories"] = np.asarray(s["trajectories"])
    return chain
