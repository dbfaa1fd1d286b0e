"""The device-resident Euler solver (detection, merge, direct passes, Euler
update on the GPU) against the reference's golden solver run and the oracle."""

from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from gpu_util import ETA_OIL, lognormal_state

pytestmark = pytest.mark.gpu


class _Post:
    stop_simulation = False

    def update_solution(self, s):
        self.solution = s

    def update_live_plot(self):
        pass

    def live_plot(self):
        pass

    def finalize_live_plot(self):
        pass


def _run(pos, r, L, dt, total_time, precision="fp64", eta_oil=ETA_OIL, eps_oil=2.85, eta_water=0.001, E=3e5,
         snapshot_depth=4, save_interval=1, correction=None, host_loop=False, graphs=True, pbm_coupling=None):
    from dem.collision_detector import SpatialHashCollisionDetector
    from dem.force_calculator import DirectDropletForceCalculator
    from dem.particle_state import DropletState
    from dem.solution import DropletSolution
    from dem.solver import EulerDropletSolver

    n = len(r)
    fc = DirectDropletForceCalculator(num_particles=n, eps_oil=eps_oil, eta_oil=eta_oil, eta_water=eta_water, E=E,
                                      L=L, boundary_mode="periodic", precision=precision,
                                      correction_grid_resolution=0 if correction is None else correction.grid_resolution)
    if correction is not None:
        fc.load_periodic_correction(correction, L_sim=L)
    det = SpatialHashCollisionDetector(num_particles=n, L=L, boundary_mode="periodic")
    sol = DropletSolution(initial_droplet_state=DropletState(pos.copy(), r.copy(), time=0.0), length=4)
    solver = EulerDropletSolver(fc, sol, _Post(), collision_detector=det, verbose=False, save_interval=save_interval,
                                snapshot_depth=snapshot_depth, graphs=graphs, pbm_coupling=pbm_coupling)
    if host_loop:
        solver._solve_host(dt, total_time)  # the reference's loop through the numpy API
    else:
        solver.solve(dt, total_time)
    chain = []
    s = solver.solution.get_first_solution()
    while s is not None:
        chain.append(s)
        s = s._next
    return solver, chain


def test_golden_solver_chain_bit_exact(golden):
    g = golden("solver_direct_periodic_n48.npz")
    _, chain = _run(g["positions"], g["radii"], float(g["L"]), float(g["dt"]), float(g["total_time"]),
                    eta_oil=float(g["eta_oil"]), eps_oil=float(g["eps_oil"]), eta_water=float(g["eta_water"]),
                    E=float(g["E"]))
    assert len(chain) == int(g["n_solutions"])
    for k, s in enumerate(chain):
        np.testing.assert_array_equal(s.radii, g[f"sol{k}_radii"])
        np.testing.assert_array_equal(s.get_times().ravel(), g[f"sol{k}_times"])
        np.testing.assert_array_equal(s.get_trajectories(), g[f"sol{k}_trajectories"])
        np.testing.assert_array_equal(np.asarray(s.collided_droplets, dtype=np.int32).reshape(-1, 2),
                                      g[f"sol{k}_collided"])


def test_lognormal_2000_twenty_steps_bit_exact():
    pos, r, L = lognormal_state(2000, seed=0)
    dt = 1e-4
    _, chain = _run(pos, r, L, dt, 19 * dt)
    ref = O.run_direct_solver(pos, r, L, True, dt, 19 * dt, eta_oil=ETA_OIL)
    assert len(chain) == len(ref)
    for s, q in zip(chain, ref):
        np.testing.assert_array_equal(s.radii, q["radii"])
        np.testing.assert_array_equal(s.get_trajectories(), q["trajectories"])


def test_mixed_trajectory_tracks_fp64():
    pos, r, L = lognormal_state(2000, seed=0)
    dt = 1e-4
    _, c64 = _run(pos, r, L, dt, 49 * dt)
    _, cmx = _run(pos, r, L, dt, 49 * dt, precision="mixed")
    assert [len(s.radii) for s in c64] == [len(s.radii) for s in cmx]
    d0 = c64[-1].get_trajectories()[-1] - c64[0].get_trajectories()[0]
    dm = cmx[-1].get_trajectories()[-1] - cmx[0].get_trajectories()[0]
    d0 -= L * np.rint(d0 / L)
    dm -= L * np.rint(dm / L)
    assert np.linalg.norm(dm - d0) <= 1e-5 * np.linalg.norm(d0)


def _same_chain(a, b):
    assert len(a) == len(b)
    for s, q in zip(a, b):
        np.testing.assert_array_equal(s.radii, q.radii)
        np.testing.assert_array_equal(s.get_times(), q.get_times())
        np.testing.assert_array_equal(s.get_trajectories(), q.get_trajectories())
        np.testing.assert_array_equal(np.asarray(s.collided_droplets).reshape(-1, 2),
                                      np.asarray(q.collided_droplets).reshape(-1, 2))


@pytest.mark.parametrize("save_interval", [1, 3])
def test_snapshot_writer_frames_equal_synchronous_frames(golden, save_interval):
    """Frames copied on the side stream (1 or 4 slots in flight) land in the same
    solutions, in the same order, with the same values as synchronous copies,
    across the six merges of the golden run."""
    g = golden("solver_direct_periodic_n48.npz")
    args = (g["positions"], g["radii"], float(g["L"]), float(g["dt"]), float(g["total_time"]))
    kw = dict(eta_oil=float(g["eta_oil"]), eps_oil=float(g["eps_oil"]), eta_water=float(g["eta_water"]),
              E=float(g["E"]), save_interval=save_interval)
    _, sync = _run(*args, snapshot_depth=0, **kw)
    for depth in (1, 4):
        solver, chain = _run(*args, snapshot_depth=depth, **kw)
        _same_chain(chain, sync)
    assert len(sync) == int(g["n_solutions"])


def test_solver_with_periodic_correction_matches_host_loop(golden):
    """The device-resident loop with the periodic-image correction (FP64)
    equals the reference's host loop driving the same calculator."""
    from dem.periodic_correction import COMSOLLatticeCorrection

    c = golden("corr_grid_comsol_r12.npz")
    corr = COMSOLLatticeCorrection.from_grid(c["grid_u"], c["grid_v"], c["grid_w"], float(c["L_comsol"]),
                                             float(c["Fz_comsol"]), float(c["eta_comsol"]))
    pos, r, L = lognormal_state(600, seed=5)
    dt = 1e-4
    _, dev = _run(pos, r, L, dt, 9 * dt, correction=corr)
    _, host = _run(pos, r, L, dt, 9 * dt, correction=corr, host_loop=True)
    _same_chain(dev, host)
    _, plain = _run(pos, r, L, dt, 9 * dt)
    assert not np.array_equal(dev[-1].get_trajectories()[-1], plain[-1].get_trajectories()[-1])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_replayed_steps_equal_eager_steps(golden, precision):
    """The step captured as a CUDA graph (per droplet count, dropped at merges)
    gives the eager step's chain bit for bit, across the golden run's merges
    and over 40 steps of a 2,000-droplet box."""
    from dem._native import launch_count

    g = golden("solver_direct_periodic_n48.npz")
    args = (g["positions"], g["radii"], float(g["L"]), float(g["dt"]), float(g["total_time"]))
    kw = dict(eta_oil=float(g["eta_oil"]), eps_oil=float(g["eps_oil"]), eta_water=float(g["eta_water"]),
              E=float(g["E"]), precision=precision)
    _, eager = _run(*args, graphs=False, **kw)
    solver, graphed = _run(*args, graphs=True, **kw)
    _same_chain(graphed, eager)
    pos, r, L = lognormal_state(2000, seed=9)
    _, eager = _run(pos, r, L, 1e-4, 39e-4, precision=precision, graphs=False)
    c0 = launch_count()
    solver, graphed = _run(pos, r, L, 1e-4, 39e-4, precision=precision, graphs=True)
    _same_chain(graphed, eager)
    assert solver.graph_replays >= 30
    assert launch_count() - c0 > 40 * 3  # replayed kernels are counted too


class _RecordingCoupling:
    """Stands in for the DEM->PBM coupling (pbm/coupling.py:51-68 upstream):
    records every on_collision(pairs, radii) and step(t, radii, dt) call with
    copies of its arguments."""

    def __init__(self):
        self.calls = []

    def on_collision(self, collided_pairs, radii):
        self.calls.append(("on_collision", np.array(collided_pairs, dtype=np.int64).copy(),
                           np.array(radii, dtype=np.float64).copy()))

    def step(self, current_time, radii, dt):
        self.calls.append(("step", float(current_time), np.array(radii, dtype=np.float64).copy(), float(dt)))


@pytest.mark.parametrize("graphs", [True, False])
def test_pbm_coupling_hooks_device_loop_equals_host_loop(golden, graphs):
    """The device-resident loop makes the same coupling calls, in the same
    order and with equal arguments, as the reference's host loop
    (euler_droplet_solver.py:100-101 on_collision before each merge,
    :135-136 step(t + dt, radii, dt) after each Euler update), across the six
    merges of the golden run."""
    g = golden("solver_direct_periodic_n48.npz")
    args = (g["positions"], g["radii"], float(g["L"]), float(g["dt"]), float(g["total_time"]))
    kw = dict(eta_oil=float(g["eta_oil"]), eps_oil=float(g["eps_oil"]), eta_water=float(g["eta_water"]),
              E=float(g["E"]))
    host, dev = _RecordingCoupling(), _RecordingCoupling()
    _, chain_h = _run(*args, host_loop=True, pbm_coupling=host, **kw)
    _, chain_d = _run(*args, graphs=graphs, pbm_coupling=dev, **kw)
    _same_chain(chain_d, chain_h)
    kinds = [c[0] for c in host.calls]
    assert kinds.count("on_collision") == int(g["n_solutions"]) - 1 >= 6
    assert kinds.count("step") >= 10
    assert len(dev.calls) == len(host.calls)
    for a, b in zip(dev.calls, host.calls):
        assert a[0] == b[0]
        if a[0] == "on_collision":
            np.testing.assert_array_equal(a[1], b[1])
            np.testing.assert_array_equal(a[2], b[2])
        else:
            assert a[1] == b[1] and a[3] == b[3]
            np.testing.assert_array_equal(a[2], b[2])
