"""Generate golden input/output vectors by running the reference's OWN ``dem/``
classes (ddkx21/particle-simulator) through the Taichi stand-in in
``tests/golden/taichi_shim``.

Run from the repository root, in a checkout where the reference is present:

    python tests/golden/make_golden.py --reference PATH   (or DEM_REFERENCE=PATH)

Every ``*.npz`` written next to this file holds the inputs, the parameters and
the reference's outputs for one case.  Tests compare the C oracle and the CUDA
path against these files; the reference itself is never needed at test time.

Cases (reference call in brackets):
  direct_*   forces + convection   [DirectDropletForceCalculator.calculate_forces_and_convection,
                                     .calculate, .calculate_convection]
  hash_*     colliding pair sets    [SpatialHashCollisionDetector.detect]
  merge_*    coalescence            [DropletSolution.generate_next_solution]
  solver_*   Euler loop with merges [EulerDropletSolver.solve]
  tree_*     flat octree            [FlatOctree.build / compute_forces_and_stokeslet /
                                     compute_forces_and_total_velocity]
  collfreq_* collision matrices     [pbm TreeCollisionFrequency.compute on a FlatOctree,
                                     DirectCollisionFrequency.compute, VolumeGrid.bin_indices]
  corr_*     periodic-image Oseen correction
                                    [COMSOLLatticeCorrection (shipped data, small grid),
                                     DirectDropletForceCalculator / FlatOctree with
                                     load_periodic_correction]
"""

from __future__ import annotations

import argparse
import contextlib
import io
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _import_reference(ref: Path):
    sys.path.insert(0, str(HERE / "taichi_shim"))
    sys.path.insert(0, str(ref))
    import taichi as ti  # the stand-in

    assert getattr(ti, "_ipow", None) is not None, "the Taichi stand-in must shadow any real taichi"
    from dem.collision_detector.spatial_hash_collision_detector import (
        SpatialHashCollisionDetector,
    )
    from dem.force_calculator.direct_droplet_force_calculator import DirectDropletForceCalculator
    from dem.octree.flat_tree import FlatOctree
    from dem.particle_state.droplet_state import DropletState
    from dem.solution.droplet_solution import DropletSolution
    from dem.solver.euler_droplet_solver import EulerDropletSolver

    from dem.periodic_correction.comsol_lattice_correction import COMSOLLatticeCorrection

    return dict(
        Corr=COMSOLLatticeCorrection,
        Ref=ref,
        Direct=DirectDropletForceCalculator,
        Hash=SpatialHashCollisionDetector,
        Tree=FlatOctree,
        State=DropletState,
        Solution=DropletSolution,
        Solver=EulerDropletSolver,
    )


# ---------------------------------------------------------------------------
# small seeded inputs
# ---------------------------------------------------------------------------
def lognormal_box(rng, n, phi=0.02, median=5e-6, sigma=0.35, gap=1e-6, periodic=True, max_tries=200):
    r = np.clip(rng.lognormal(np.log(median), sigma, n), 1e-6, 30e-6)
    L = float(np.cbrt(np.sum(4.0 / 3.0 * np.pi * r**3) / phi))
    pos = rng.uniform(0.0, L, (n, 3))
    for _ in range(max_tries):
        d = pos[None, :, :] - pos[:, None, :]
        if periodic:
            d -= L * np.rint(d / L)
        dist = np.sqrt((d**2).sum(-1))
        np.fill_diagonal(dist, np.inf)
        bad = np.triu(dist < (r[:, None] + r[None, :] + gap))
        ii, jj = np.nonzero(bad)
        if len(ii) == 0:
            break
        redo = np.unique(jj)
        pos[redo] = rng.uniform(0.0, L, (len(redo), 3))
    return pos, r, L


def dense_box(rng, n, L, rmin, rmax):
    return rng.uniform(0.0, L, (n, 3)), rng.uniform(rmin, rmax, n)


# ---------------------------------------------------------------------------
# cases
# ---------------------------------------------------------------------------
PHYS = dict(eps_oil=2.85, eta_oil=0.06, eta_water=0.001, E=3e5)


def gen_direct(R, out):
    rng = np.random.default_rng(11)
    cases = []
    pos, r, L = lognormal_box(rng, 96)
    cases.append(("direct_periodic_n96", pos, r, L, "periodic"))
    pos, r, L = lognormal_box(rng, 64, periodic=False)
    cases.append(("direct_open_n64", pos, r, L, "open"))
    # dense: many pairs inside the contact cut (r_ij <= r_i + r_j) and near contact
    pos, r = dense_box(rng, 48, 2e-4, 5e-6, 30e-6)
    cases.append(("direct_contact_n48", pos, r, 2e-4, "periodic"))
    # reference default box (L=1 m, periodic), droplets in a corner and across the faces
    pos = rng.uniform(0.0, 1.0, (24, 3)) * np.array([1.0, 1.0, 1.0])
    r = rng.uniform(1e-2, 4e-2, 24)
    cases.append(("direct_unitbox_n24", pos, r, 1.0, "periodic"))
    # hand-made two-body and three-body configurations
    two = np.array(
        [
            [0.40, 0.50, 0.50],
            [0.60, 0.50, 0.50],  # along x
            [0.50, 0.50, 0.40],
            [0.50, 0.50, 0.60],  # along z
            [0.05, 0.50, 0.50],
            [0.95, 0.51, 0.52],  # across the periodic face in x
        ]
    )
    cases.append(("direct_fewbody_n6", two, np.array([2e-2, 2e-2, 1e-2, 3e-2, 1e-2, 1e-2]), 1.0, "periodic"))
    for name, pos, r, L, mode in cases:
        n = len(r)
        fc = R["Direct"](num_particles=n, L=L, boundary_mode=mode, **PHYS)
        F, V = fc.calculate_forces_and_convection(pos, r)
        F1 = fc.calculate(pos, r)
        V1 = fc.calculate_convection(pos, r, F1)
        assert np.array_equal(F, F1) and np.array_equal(V, V1)
        np.savez(
            out / f"{name}.npz",
            positions=pos,
            radii=r,
            L=L,
            periodic=int(mode == "periodic"),
            m_const=fc.m_const,
            eta_const=fc.eta_const,
            forces=F,
            velocities=V,
            **{k: v for k, v in PHYS.items()},
        )
        print(f"{name}: n={n} |F|max={np.abs(F).max():.3e} |V|max={np.abs(V).max():.3e}")


def gen_hash(R, out):
    rng = np.random.default_rng(12)
    cases = []
    pos, r = dense_box(rng, 300, 1e-3, 20e-6, 60e-6)
    cases.append(("hash_dense_periodic_n300", pos, r, 1e-3, "periodic"))
    cases.append(("hash_dense_open_n300", pos, r, 1e-3, "open"))
    # grid_dim = 2 and 3: neighbour cells alias after the periodic wrap
    pos, r = dense_box(rng, 40, 1e-3, 150e-6, 200e-6)
    cases.append(("hash_tinygrid_periodic_n40", pos, r, 1e-3, "periodic"))
    pos, r = dense_box(rng, 60, 1e-3, 100e-6, 160e-6)
    cases.append(("hash_grid3_periodic_n60", pos, r, 1e-3, "periodic"))
    # partial last cell: L not a multiple of the cell size
    pos, r = dense_box(rng, 400, 1e-3, 10e-6, 37e-6)
    cases.append(("hash_partialcell_periodic_n400", pos, r, 1e-3, "periodic"))
    # positions outside [0, L) in open mode (clamped cells)
    pos = rng.uniform(-2e-4, 1.2e-3, (200, 3))
    r = rng.uniform(10e-6, 40e-6, 200)
    cases.append(("hash_outside_open_n200", pos, r, 1e-3, "open"))
    # a lognormal 2 % box, as in the measured configurations
    pos, r, L = lognormal_box(rng, 512, gap=-3e-6)  # negative gap lets some droplets touch
    cases.append(("hash_lognormal_periodic_n512", pos, r, L, "periodic"))
    for name, pos, r, L, mode in cases:
        n = len(r)
        det = R["Hash"](num_particles=4 * n, L=L, boundary_mode=mode)  # room for every pair
        flag, pairs = det.detect(pos, r)
        table = det._hash_table_size
        np.savez(
            out / f"{name}.npz",
            positions=pos,
            radii=r,
            L=L,
            periodic=int(mode == "periodic"),
            table_size=table,
            capacity=4 * n,
            is_collision=int(flag),
            pairs=pairs.astype(np.int32),
        )
        print(f"{name}: n={n} pairs={len(pairs)} table={table}")


def gen_merge(R, out):
    rng = np.random.default_rng(13)
    cases = []
    pos = np.array([[0.0, 0.0, 0.0], [0.1, 0.0, 0.0], [0.5, 0.5, 0.5]])
    cases.append(("merge_three_to_two", pos, np.array([0.05, 0.05, 0.05]), np.array([[0, 1]])))
    # chains: 0-1, 1-2, 2-3 (greedy takes 0-1 and 2-3), a star around 5, an isolated pair
    n = 12
    pos = rng.uniform(0, 1e-3, (n, 3))
    r = rng.uniform(5e-6, 20e-6, n)
    pairs = np.array([[0, 1], [1, 2], [2, 3], [5, 6], [5, 7], [5, 9], [6, 7], [8, 11], [10, 11]])
    cases.append(("merge_chains_n12", pos, r, pairs))
    # pairs from a real detection
    pos, r = dense_box(rng, 200, 1e-3, 15e-6, 45e-6)
    det = R["Hash"](num_particles=800, L=1e-3, boundary_mode="periodic")
    _, pairs = det.detect(pos, r)
    cases.append(("merge_detected_n200", pos, r, pairs))
    for name, pos, r, pairs in cases:
        pairs = np.asarray(pairs, dtype=np.int32).reshape(-1, 2)
        # the reference orders by column 0 with np.argsort; make sure the case does not
        # depend on how ties are broken
        assert np.array_equal(np.argsort(pairs[:, 0]), np.argsort(pairs[:, 0], kind="stable"))
        st = R["State"](pos.copy(), r.copy(), time=0.25)
        sol = R["Solution"](initial_droplet_state=st, length=4)
        sol.collided_droplets = pairs.copy()
        with contextlib.redirect_stdout(io.StringIO()):
            nxt = sol.generate_next_solution()
        np.savez(
            out / f"{name}.npz",
            positions=pos,
            radii=r,
            pairs=pairs,
            new_positions=nxt.initial_droplet_state.positions,
            new_radii=nxt.initial_droplet_state.radii,
        )
        print(f"{name}: n={len(r)} -> {len(nxt.radii)}")


class _StubPost:
    stop_simulation = False

    def update_solution(self, s):
        self.solution = s

    def update_live_plot(self):
        pass

    def live_plot(self):
        pass

    def finalize_live_plot(self):
        pass


def gen_solver(R, out):
    rng = np.random.default_rng(14)
    n = 48
    pos, r, L = lognormal_box(rng, n, phi=0.06, gap=0.5e-6)
    # put a few droplets almost in contact along the field (z): they attract and merge
    for k in range(0, 12, 2):
        pos[k + 1] = pos[k] + np.array([0.0, 0.0, r[k] + r[k + 1] + 0.3e-6 * (1 + k)])
    pos %= L
    dt, steps = 0.02, 12
    fc = R["Direct"](num_particles=n, L=L, boundary_mode="periodic", **PHYS)
    det = R["Hash"](num_particles=n, L=L, boundary_mode="periodic")
    st = R["State"](pos.copy(), r.copy(), time=0.0)
    sol = R["Solution"](initial_droplet_state=st, length=4)
    solver = R["Solver"](fc, sol, _StubPost(), collision_detector=det)
    with contextlib.redirect_stdout(io.StringIO()):
        solver.solve(dt, dt * (steps - 1))  # the reference runs int(T/dt)+1 steps
    first = solver.solution.get_first_solution()
    chain = []
    s = first
    while s is not None:
        chain.append(s)
        s = s._next
    payload = dict(
        positions=pos,
        radii=r,
        L=L,
        dt=dt,
        total_time=dt * (steps - 1),
        stokes_factor=solver.stokes_factor,
        n_solutions=len(chain),
        **{k: v for k, v in PHYS.items()},
    )
    for k, s in enumerate(chain):
        payload[f"sol{k}_radii"] = np.asarray(s.radii)
        payload[f"sol{k}_times"] = np.asarray(s.get_times()).ravel()
        payload[f"sol{k}_trajectories"] = np.asarray(s.get_trajectories())
        cd = np.asarray(s.collided_droplets, dtype=np.int32).reshape(-1, 2)
        payload[f"sol{k}_collided"] = cd
    np.savez(out / "solver_direct_periodic_n48.npz", **payload)
    print(f"solver: {len(chain)} solutions, final n={len(chain[-1].radii)}, steps={steps}")


def gen_tree(R, out):
    rng = np.random.default_rng(15)
    base_pos, base_r, base_L = lognormal_box(rng, 160, phi=0.05)
    cases = [
        ("tree_open_mpl1_t05_n160", base_pos, base_r, base_L, False, 0.5, 1),
        ("tree_periodic_mpl4_t05_n160", base_pos, base_r, base_L, True, 0.5, 4),
        ("tree_periodic_mpl1_t03_n160", base_pos, base_r, base_L, True, 0.3, 1),
    ]
    pos, r = dense_box(rng, 120, 1e-2, 20e-6, 50e-6)
    cases.append(("tree_open_mpl2_t08_n120", pos, r, 1e-2, False, 0.8, 2))
    # clustered: many droplets in one corner forces deep levels
    pos = np.concatenate([rng.uniform(0, 1e-4, (60, 3)), rng.uniform(0, 1e-2, (40, 3))])
    r = rng.uniform(1e-6, 3e-6, 100)
    cases.append(("tree_cluster_mpl1_t05_n100", pos, r, 1e-2, False, 0.5, 1))
    m_const = 12 * np.pi * 8.85418781762039e-12 * PHYS["eps_oil"] * PHYS["E"] ** 2
    eta_const = 1 / (8 * np.pi * PHYS["eta_oil"])
    sf = 2 * np.pi * PHYS["eta_oil"] * (2 * PHYS["eta_oil"] + 3 * PHYS["eta_water"]) / (
        PHYS["eta_oil"] + PHYS["eta_water"]
    )
    for name, pos, r, L, periodic, theta, mpl in cases:
        n = len(r)
        t = R["Tree"](theta=theta, mpl=mpl, num_particles=n)
        t.build(pos, r, L, periodic)
        F, V = t.compute_forces_and_stokeslet(m_const, eta_const)
        F, V = F.copy(), V.copy()
        t.build(pos, r, L, periodic)
        F2, VT = t.compute_forces_and_total_velocity(m_const, eta_const, sf)
        F2, VT = F2.copy(), VT.copy()
        assert np.array_equal(F, F2)
        count = t.nodes.count.to_numpy()[: t.node_count[None]]
        first_child = t.nodes.first_child.to_numpy()[: t.node_count[None]]
        np.savez(
            out / f"{name}.npz",
            positions=pos,
            radii=r,
            L=L,
            periodic=int(periodic),
            theta=theta,
            mpl=mpl,
            m_const=m_const,
            eta_const=eta_const,
            stokes_factor=sf,
            node_count=t.node_count[None],
            parent_count=t.parent_count[None],
            leaf_slot_count=t.leaf_slot_count[None],
            max_nodes=t.max_nodes,
            node_counts=count,
            node_is_leaf=(first_child < 0).astype(np.int8),
            forces=F,
            velocities=V,
            total_velocities=VT,
        )
        print(f"{name}: nodes={t.node_count[None]} parents={t.parent_count[None]}")


def _synthetic_correction(R, rng, n, L_comsol, Fz, eta):
    """A COMSOLLatticeCorrection whose regular grid is a seeded smooth field with
    no symmetry (exercises every corner weight, the clamping and the permuted
    lookups); built around the reference's own evaluate()."""
    c = object.__new__(R["Corr"])
    c.L_comsol, c.Fz_comsol, c.eta_comsol, c.grid_resolution = L_comsol, Fz, eta, n
    c.grid_coords = np.linspace(-L_comsol / 2, L_comsol / 2, n)
    g = np.meshgrid(c.grid_coords, c.grid_coords, c.grid_coords, indexing="ij")
    fields = []
    for k in range(3):
        a = rng.normal(size=(4, 3))
        f = sum(a[m, 0] * np.sin((m + 1) * 2.1 * g[0] / L_comsol + a[m, 1]) * np.cos((m + 2) * 1.7 * g[1] / L_comsol)
                * np.cos(m * 2.9 * g[2] / L_comsol + a[m, 2]) for m in range(4))
        fields.append(1e-9 * (f + 0.05 * rng.normal(size=f.shape)))
    c.grid_u, c.grid_v, c.grid_w = fields
    c._interp_u, c._interp_v, c._interp_w = c._build_interpolators()
    return c


def gen_correction(R, out):
    rng = np.random.default_rng(16)
    data = Path(R["Ref"]) / "dem" / "periodic_correction" / "data"
    import json

    prm = json.loads((data / "comsol_params.json").read_text())
    Fz = 4 * np.pi * prm["R"] ** 2 * prm["eps_0"] * prm["eps_r"] * prm["E0"] ** 2  # comsol_lattice_correction.py:46
    with contextlib.redirect_stdout(io.StringIO()):
        comsol = R["Corr"](data_path=str(data / prm["velocity_file"]), L_comsol=prm["L"], Fz_comsol=Fz,
                           eta_comsol=prm["eta"], grid_resolution=12)
    gd = comsol.get_grid_data()
    probe = rng.uniform(-0.6, 0.6, (40, 3)) * prm["L"]  # some outside the cell (fill value 0)
    probe_F = rng.normal(size=(40, 3)) * 1e-9
    np.savez(out / "corr_grid_comsol_r12.npz", **{k: gd[k] for k in gd}, probe=probe, probe_F=probe_F,
             eval_raw=comsol.evaluate(probe), eval_F=comsol.evaluate(probe, probe_F),
             eval_origin=comsol.evaluate(np.zeros((1, 3))))
    print(f"corr_grid_comsol_r12: |w|max={np.abs(gd['grid_w']).max():.3e}")
    synth = _synthetic_correction(R, rng, 7, 2e-4, 3.3e-12, 0.05)

    def save_grid(payload, c):
        g = c.get_grid_data()
        payload.update(grid_u=g["grid_u"], grid_v=g["grid_v"], grid_w=g["grid_w"], grid_min=g["grid_min"],
                       grid_dx=g["grid_dx"], grid_resolution=g["grid_resolution"], L_comsol=g["L_comsol"],
                       Fz_comsol=g["Fz_comsol"], eta_comsol=g["eta_comsol"])

    # direct: shipped data (periodic) and the synthetic grid (periodic, open: clamped lookups)
    pos, r, L = lognormal_box(rng, 64)
    pos2, r2, L2 = lognormal_box(rng, 40, periodic=False)
    for name, c, pos, r, L, mode in (("corr_direct_comsol_periodic_n64", comsol, pos, r, L, "periodic"),
                                     ("corr_direct_synth_periodic_n64", synth, pos, r, L, "periodic"),
                                     ("corr_direct_synth_open_n40", synth, pos2, r2, L2, "open")):
        n = len(r)
        fc = R["Direct"](num_particles=n, L=L, boundary_mode=mode, correction_grid_resolution=c.grid_resolution,
                         **PHYS)
        with contextlib.redirect_stdout(io.StringIO()):
            fc.load_periodic_correction(c, L_sim=L)
        F, V = fc.calculate_forces_and_convection(pos, r)
        payload = dict(positions=pos, radii=r, L=L, periodic=int(mode == "periodic"), m_const=fc.m_const,
                       eta_const=fc.eta_const, eta_oil=fc.eta_oil, forces=F, velocities=V,
                       corr_self_coeff=fc.corr_self_coeff[None], corr_L_ratio=fc.corr_L_ratio[None],
                       corr_eta_ratio=fc.corr_eta_ratio[None], corr_Fz_inv=fc.corr_Fz_inv[None])
        save_grid(payload, c)
        np.savez(out / f"{name}.npz", **payload)
        print(f"{name}: n={n} |V|max={np.abs(V).max():.3e} self={fc.corr_self_coeff[None]:.3e}")

    # tree: Stokeslet and total-velocity walks with the correction at leaf pairs and accepted nodes
    m_const = 12 * np.pi * 8.85418781762039e-12 * PHYS["eps_oil"] * PHYS["E"] ** 2
    eta_const = 1 / (8 * np.pi * PHYS["eta_oil"])
    sf = 2 * np.pi * PHYS["eta_oil"] * (2 * PHYS["eta_oil"] + 3 * PHYS["eta_water"]) / (
        PHYS["eta_oil"] + PHYS["eta_water"]
    )
    pos, r, L = lognormal_box(rng, 120, phi=0.05)
    for name, c, periodic, theta, mpl in (("corr_tree_comsol_periodic_mpl2_t05_n120", comsol, True, 0.5, 2),
                                          ("corr_tree_synth_open_mpl1_t07_n120", synth, False, 0.7, 1)):
        n = len(r)
        t = R["Tree"](theta=theta, mpl=mpl, num_particles=n, correction_grid_resolution=c.grid_resolution)
        t.load_periodic_correction(c, L, eta_sim=PHYS["eta_oil"])
        t.build(pos, r, L, periodic)
        F, V = t.compute_forces_and_stokeslet(m_const, eta_const)
        F, V = F.copy(), V.copy()
        t.build(pos, r, L, periodic)
        F2, VT = t.compute_forces_and_total_velocity(m_const, eta_const, sf)
        VT = VT.copy()
        assert np.array_equal(F, F2)
        payload = dict(positions=pos, radii=r, L=L, periodic=int(periodic), theta=theta, mpl=mpl, m_const=m_const,
                       eta_const=eta_const, eta_oil=PHYS["eta_oil"], stokes_factor=sf, forces=F, velocities=V,
                       total_velocities=VT, corr_self_coeff=t.corr_self_coeff[None],
                       corr_L_ratio=t.corr_L_ratio[None], corr_eta_ratio=t.corr_eta_ratio[None],
                       corr_Fz_inv=t.corr_Fz_inv[None])
        save_grid(payload, c)
        np.savez(out / f"{name}.npz", **payload)
        print(f"{name}: nodes={t.node_count[None]} |V|max={np.abs(V).max():.3e}")


def gen_collfreq(R, out):
    from pbm.collision_frequency import DirectCollisionFrequency, TreeCollisionFrequency
    from pbm.volume_grid import VolumeGrid

    rng = np.random.default_rng(17)
    cases = []
    # the reference's own test configurations (tests/pbm/collision_frequency/test_tree_collision_freq.py)
    pos = np.array([[0.10, 0.10, 0.10], [0.12, 0.10, 0.10], [0.50, 0.50, 0.50], [0.80, 0.10, 0.10],
                    [0.10, 0.80, 0.10], [0.10, 0.10, 0.80]])
    cases.append(("collfreq_reftest_n6", pos, np.full(6, 0.025), 1.0, False, (0.01, 0.05, 4, "geometric"), 1))
    pos = np.array([[0.01, 0.5, 0.5], [0.99, 0.5, 0.5]])
    cases.append(("collfreq_periodic_n2", pos, np.full(2, 0.05), 1.0, True, (0.02, 0.1, 3, "geometric"), 1))
    # dense boxes with many contacts, mixed sizes (some outside the grid: clamped bins)
    pos, r = dense_box(rng, 400, 1e-3, 10e-6, 45e-6)
    cases.append(("collfreq_dense_periodic_n400", pos, r, 1e-3, True, (12e-6, 40e-6, 6, "geometric"), 2))
    cases.append(("collfreq_dense_open_n400", pos, r, 1e-3, False, (12e-6, 40e-6, 5, "linear"), 4))
    for name, pos, r, L, periodic, (rmin, rmax, nb, spacing), mpl in cases:
        n = len(r)
        g = VolumeGrid.from_radii_range(rmin, rmax, nb, spacing)
        tree = R["Tree"](theta=0.5, mpl=mpl, num_particles=n)
        tree.build(pos, r, L, periodic)
        M_tree = TreeCollisionFrequency(tree, g, max_particles=n).compute(pos, r)
        M_direct = DirectCollisionFrequency(g).compute(pos, r, L=L, periodic=periodic)
        bins = g.bin_indices((4.0 / 3.0) * np.pi * r**3)
        np.savez(out / f"{name}.npz", positions=pos, radii=r, L=L, periodic=int(periodic), mpl=mpl, r_min=rmin,
                 r_max=rmax, n_bins=nb, spacing=spacing, bins=bins.astype(np.int32), edges=g.edges,
                 matrix_tree=M_tree, matrix_direct=M_direct)
        print(f"{name}: pairs={int(M_tree.sum()) // 2} same_as_direct={np.array_equal(M_tree, M_direct)}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("DEM_REFERENCE"),
                    help="the reference checkout (default: $DEM_REFERENCE)")
    ap.add_argument("--only", default="")
    args = ap.parse_args()
    if not args.reference:
        ap.error("name the reference checkout with --reference or DEM_REFERENCE")
    R = _import_reference(Path(args.reference))
    gens = dict(direct=gen_direct, hash=gen_hash, merge=gen_merge, solver=gen_solver, tree=gen_tree,
                correction=gen_correction, collfreq=gen_collfreq)
    for k, g in gens.items():
        if args.only and k not in args.only.split(","):
            continue
        g(R, HERE)


if __name__ == "__main__":
    main()
