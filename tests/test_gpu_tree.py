"""Flat octree on the GPU against the reference's golden vectors and the
oracle: identical tree structure, bit-identical forces and velocities."""

from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN
from gpu_util import ETA_OIL, consts, lognormal_state

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(p.name for p in GOLDEN.glob("tree_*.npz")))
def test_tree_bit_exact_against_golden(golden, name):
    from dem.octree import FlatOctree

    g = golden(name)
    t = FlatOctree(theta=float(g["theta"]), mpl=int(g["mpl"]), num_particles=len(g["radii"]))
    assert t.max_nodes == int(g["max_nodes"])
    t.build(g["positions"], g["radii"], L=float(g["L"]), periodic=bool(g["periodic"]))
    assert t.node_count[None] == int(g["node_count"])
    assert t.parent_count[None] == int(g["parent_count"])
    assert t.leaf_slot_count[None] == int(g["leaf_slot_count"])
    np.testing.assert_array_equal(t.nodes.count.to_numpy(), g["node_counts"])
    np.testing.assert_array_equal((t.nodes.first_child.to_numpy() < 0).astype(np.int8), g["node_is_leaf"])
    F, V = t.compute_forces_and_stokeslet(float(g["m_const"]), float(g["eta_const"]))
    np.testing.assert_array_equal(F, g["forces"])
    np.testing.assert_array_equal(V, g["velocities"])
    t.build(g["positions"], g["radii"], L=float(g["L"]), periodic=bool(g["periodic"]))
    F2, VT = t.compute_forces_and_total_velocity(float(g["m_const"]), float(g["eta_const"]), float(g["stokes_factor"]))
    np.testing.assert_array_equal(F2, g["forces"])
    np.testing.assert_array_equal(VT, g["total_velocities"])


@pytest.mark.parametrize("n,mpl,theta,periodic,max_nodes", [
    (20000, 4, 0.5, True, None),
    (20000, 16, 0.5, True, None),
    (6000, 1, 0.3, False, None),
    (8000, 1, 0.5, True, 4000),  # node pool exhausted: subdivision stops in node order
])
def test_tree_bit_exact_against_oracle(n, mpl, theta, periodic, max_nodes):
    from dem.octree import FlatOctree

    pos, r, L = lognormal_state(n, seed=n % 7, periodic=periodic)
    m, eta, sf = consts()
    t = FlatOctree(theta=theta, mpl=mpl, num_particles=n, max_nodes=max_nodes)
    t.build(pos, r, L=L, periodic=periodic)
    ref = O.Tree(n, theta, mpl, max_nodes=max_nodes or 0)
    ref.build(pos, r, L, periodic)
    st = ref.stats()
    assert t.node_count[None] == st["node_count"]
    assert t.parent_count[None] == st["parent_count"]
    assert t.leaf_slot_count[None] == st["leaf_slot_count"]
    nd = ref.nodes()
    np.testing.assert_array_equal(t.nodes.count.to_numpy(), nd["count"])
    np.testing.assert_array_equal(t.nodes.first_child.to_numpy(), nd["first_child"])
    np.testing.assert_array_equal(t.nodes.next.to_numpy(), nd["next"])
    np.testing.assert_array_equal(t.leaf_indices.to_numpy(), ref.leaf_indices())
    F, VT = t.compute_forces_and_total_velocity(m, eta, sf)
    F_ref, VT_ref = ref.forces_and_total_velocity(m, eta, sf)
    np.testing.assert_array_equal(F, F_ref)
    np.testing.assert_array_equal(VT, VT_ref)
    if max_nodes:
        assert t._tree.stats()["pool_exhausted"] == 1


def test_stokeslet_with_given_forces():
    from dem.octree import FlatOctree

    pos, r, L = lognormal_state(3000, seed=4)
    m, eta, _ = consts()
    rng = np.random.default_rng(0)
    F_in = rng.normal(size=(3000, 3)) * 1e-12
    t = FlatOctree(theta=0.5, mpl=2, num_particles=3000)
    t.build(pos, r, L=L, periodic=True)
    V = t.compute_stokeslet(F_in, eta)
    ref = O.Tree(3000, 0.5, 2)
    ref.build(pos, r, L, True)
    ref.propagate_forces(F_in)
    np.testing.assert_array_equal(V, ref.velocity(F_in, eta))


def test_reference_tree_invariants():
    # tests/octree/test_flat_tree.py and test_force_tree.py upstream
    from dem.force_calculator import DirectDropletForceCalculator
    from dem.octree import FlatOctree, TreeDropletForceCalculator

    rng = np.random.default_rng(42)
    pos = rng.random((50, 3))
    t = FlatOctree(theta=0.5, mpl=1, num_particles=50)
    t.build(pos, rng.random(50) * 0.005 + 0.005, L=1.0, periodic=False)
    assert t.nodes.count.to_numpy()[0] == 50 and t.num_particles[None] == 50
    rng = np.random.default_rng(0)
    pos = rng.random((80, 3))
    counts = []
    for mpl in (8, 1):
        t = FlatOctree(theta=0.5, mpl=mpl, num_particles=80)
        t.build(pos, np.full(80, 0.005), L=1.0, periodic=False)
        counts.append(int(t.node_count[None]))
    assert counts[1] > counts[0]
    t = FlatOctree(theta=0.5, mpl=1, num_particles=16)
    t.update_params(theta=0.3, mpl=4)
    assert t.theta == 0.3 and t.mpl == 4 and t.theta_sq[None] == 0.3 * 0.3 and t.mpl_field[None] == 4
    t = FlatOctree(theta=0.5, mpl=1, num_particles=10)
    p = np.random.default_rng(1).random((10, 3))
    t.build(p, np.full(10, 0.01), L=1.0, periodic=False)
    assert t.periodic[None] == 0
    t.build(p, np.full(10, 0.01), L=1.0, periodic=True)
    assert t.periodic[None] == 1
    with pytest.raises(ValueError):
        FlatOctree(num_particles=10).build(np.zeros((100, 3)), np.ones(100), L=1.0)

    def rel(a, b):
        d = np.linalg.norm(a - b, axis=1)
        ref = np.linalg.norm(a, axis=1) + np.mean(np.linalg.norm(a, axis=1)) * 1e-10
        return d / ref

    rng = np.random.default_rng(42)
    n, L = 30, 0.01
    pos = rng.random((n, 3)) * L
    radii = rng.random(n) * 30e-6 + 20e-6
    d = DirectDropletForceCalculator(num_particles=n, L=L, boundary_mode="open")
    f_d = d.calculate(pos, radii)
    v_d = d.calculate_convection(pos, radii, f_d)
    tr = TreeDropletForceCalculator(num_particles=n, theta=0.3, mpl=1, L=L, periodic=False)
    f_t = tr.calculate(pos, radii)
    v_t = tr.calculate_convection(pos, radii, f_t)
    assert np.mean(rel(f_d, f_t)) < 0.05
    assert np.mean(rel(v_d, v_t)) < 0.1
    prev = float("inf")
    for theta in (0.8, 0.5, 0.3):
        tr = TreeDropletForceCalculator(num_particles=n, theta=theta, mpl=1, L=L, periodic=False)
        err = float(np.mean(rel(f_d, tr.calculate(pos, radii))))
        assert err <= prev + 1e-4
        prev = err


def test_tree_solver_device_path_matches_oracle():
    """EulerDropletSolver with the tree calculator (device-resident loop) against
    the oracle tree driven with the reference's loop (euler_droplet_solver.py:113-131)."""
    from dem.octree import TreeDropletForceCalculator
    from dem.particle_state import DropletState
    from dem.solution import DropletSolution
    from dem.solver import EulerDropletSolver

    class Post:
        stop_simulation = False

        def update_solution(self, s):
            pass

        def live_plot(self):
            pass

        def update_live_plot(self):
            pass

        def finalize_live_plot(self):
            pass

    pos, r, L = lognormal_state(4000, seed=3)
    m, eta, sf = consts()
    dt = 1e-4
    fc = TreeDropletForceCalculator(num_particles=4000, theta=0.5, mpl=4, eta_oil=ETA_OIL, L=L, periodic=True)
    sol = DropletSolution(DropletState(pos.copy(), r.copy(), 0.0), length=8)
    solver = EulerDropletSolver(fc, sol, Post(), collision_detector=None, verbose=False)
    solver.solve(dt, 4 * dt)
    got = solver.solution.get_trajectories()
    ref = O.Tree(4000, 0.5, 4)
    p = pos.copy()
    frames = [p.copy()]
    for _ in range(solver.steps_taken):
        ref.build(p, r, L, True)
        _, VT = ref.forces_and_total_velocity(m, eta, sf)
        p = O.euler_total(p, VT, dt, L, True)
        frames.append(p.copy())
    np.testing.assert_array_equal(got, np.asarray(frames))
