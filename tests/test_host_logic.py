"""Host-side logic that needs no GPU: the reference's own solver and solution
tests (tests/solver/test_euler_droplet_solver.py, tests/solution/
test_droplet_solution.py upstream) run against the drop-in classes with the
same stubs, plus helpers of the detector and the merge."""

from __future__ import annotations

from dataclasses import dataclass
from pathlib import Path

import numpy as np
import pytest

from dem.collision_detector.spatial_hash_collision_detector import _next_power_of_2
from dem.particle_generator import LognormalDropletGenerator, box_side_for_volume_fraction
from dem.particle_state import DropletState
from dem.solution import DropletSolution
from dem.solution.droplet_solution import order_pairs
from dem.solver import EulerDropletSolver


@dataclass
class StubForceCalculator:
    F: float = 1e-12
    L: float = 1.0
    eta_oil: float = 0.065
    eta_water: float = 0.001
    boundary_mode: str = "open"

    def calculate_forces_and_convection(self, positions, radii):
        n = len(radii)
        forces = np.zeros((n, 3))
        forces[:, 2] = self.F
        return forces, np.zeros((n, 3))


class StubPostProcessor:
    def __init__(self):
        self.stop_simulation = False
        self.live_calls = 0

    def update_solution(self, s):
        self.solution = s

    def update_live_plot(self):
        self.live_calls += 1

    def live_plot(self):
        self.live_calls += 1

    def finalize_live_plot(self):
        pass


def _make_solver(F=1e-12, n=2):
    state = DropletState(np.zeros((n, 3)), np.full(n, 50e-6), time=0.0)
    sol = DropletSolution(initial_droplet_state=state, length=20)
    return EulerDropletSolver(force_calculator=StubForceCalculator(F=F), solution=sol,
                              post_processor=StubPostProcessor(), verbose=False)


def test_stokes_factor_positive():
    assert _make_solver().stokes_factor > 0


def test_drops_move_in_z():
    s = _make_solver(F=1e-12)
    s.solve(dt=1e-3, total_time=1e-2)
    p = s.solution.get_current_positions()
    assert np.all(p[:, 2] > 0)
    np.testing.assert_allclose(p[:, 0], 0.0)
    np.testing.assert_allclose(p[:, 1], 0.0)


def test_time_advances_and_step_count():
    s = _make_solver()
    s.solve(dt=1e-3, total_time=5e-3)
    assert s.solution.get_current_time() > 0
    # int(T/dt) + 1 steps, like the reference
    assert s.steps_taken == int(5e-3 / 1e-3) + 1


def test_stop_simulation():
    s = _make_solver()
    s.post_processor.stop_simulation = True
    s.solve(dt=1e-3, total_time=1.0)
    assert s.solution.current_step == 0


def test_periodic_wrap():
    s = _make_solver(F=1e-9)
    s.force_calculator.boundary_mode = "periodic"
    s.force_calculator.L = 0.001
    s.solve(dt=1e-4, total_time=1e-3)
    p = s.solution.get_current_positions()
    assert np.all(p[:, 2] >= 0) and np.all(p[:, 2] < 0.001)


def test_solution_buffers_and_accessors(tmp_path: Path):
    rng = np.random.default_rng(0)
    st = DropletState(rng.random((3, 3)), np.full(3, 0.05), time=0.0)
    sol = DropletSolution(initial_droplet_state=st, length=2)
    for k in range(5):
        sol.save_step(k * 0.1, np.full((3, 3), float(k)))
    assert sol.length >= 6
    t = sol.get_times().ravel()
    assert t[-1] >= t[0]
    sol.compact()
    assert len(sol.times) == sol.current_step + 1
    path = tmp_path / "chain.npz"
    sol.save_chain_to_file(str(path))
    loaded = DropletSolution.load_chain_from_file(str(path))
    np.testing.assert_allclose(loaded.radii, sol.radii)
    np.testing.assert_allclose(loaded.trajectories, sol.get_trajectories())


def test_get_state_interpolates():
    rng = np.random.default_rng(0)
    st = DropletState(rng.random((3, 3)), np.full(3, 0.05), time=0.0)
    sol = DropletSolution(initial_droplet_state=st, length=5)
    sol.save_step(1.0, np.full((3, 3), 1.0))
    sol.compact()
    mid = sol.get_state(0.5)
    np.testing.assert_allclose(mid.positions, (st.positions + 1.0) / 2)
    with pytest.raises(ValueError):
        sol.get_state(-1.0)


@pytest.mark.parametrize("n,expected", [(1, 1), (2, 2), (3, 4), (5, 8), (16, 16), (17, 32)])
def test_next_power_of_2(n, expected):
    assert _next_power_of_2(n) == expected


def test_order_pairs_is_stable_by_first_index():
    p = order_pairs([[3, 4], [1, 9], [1, 2], [0, 5]])
    np.testing.assert_array_equal(p, [[0, 5], [1, 9], [1, 2], [3, 4]])


def test_lognormal_generator_is_seeded_and_overlap_free():
    a = LognormalDropletGenerator(400, seed=3).generate()
    b = LognormalDropletGenerator(400, seed=3).generate()
    np.testing.assert_array_equal(a.positions, b.positions)
    g = LognormalDropletGenerator(400, seed=3)
    s = g.generate()
    L = g.L
    assert abs(L - box_side_for_volume_fraction(s.radii, 0.02)) < 1e-15
    d = s.positions[:, None, :] - s.positions[None, :, :]
    d -= L * np.rint(d / L)
    dist = np.sqrt((d**2).sum(-1))
    np.fill_diagonal(dist, np.inf)
    assert np.all(dist >= s.radii[:, None] + s.radii[None, :] + 1e-6 - 1e-18)
    assert s.radii.min() >= 1e-6 and s.radii.max() <= 30e-6
