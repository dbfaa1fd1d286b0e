"""Explicit Euler solver of the droplet system.

Drop-in for dem/solver/euler_droplet_solver.py:8-159 of
ddkx21/particle-simulator: same constructor, attributes and loop semantics:

* before every step the colliding pairs are detected; on a collision the
  droplets are merged, a new solution is chained at the same time and the
  detection is repeated (time does not advance);
* ``remaining_steps = int((t_end - t) / dt) + 1`` steps per pass (:74), so a
  run may overshoot ``t_end`` by up to one step, like the reference;
* v = F / (stokes_factor r) + v_conv (direct) or the tree's total velocity;
  x += v dt; x %= L in periodic mode.

When the force calculator and the detector are the B200 classes of this
package, the state stays on the device for the whole run: detection, merge,
both O(N^2) passes and the Euler update are CUDA kernels, and only the pair
count (every step), the saved trajectory frames and the merged state cross
PCIe.  With the direct calculator a step runs speculatively: detection, forces,
convection and the Euler update into the other position buffer are one CUDA
graph (captured once per droplet count and replayed), followed by one read of
the pair count; when pairs were found the new positions are dropped and the
merge proceeds from the unchanged ones, as in the reference.  Saved
frames are copied on a separate stream into pinned host slots
(``dem.solution.snapshot.SnapshotWriter``) while the next steps run, and are
appended to the solution in order.  Any other (duck-typed) calculator or
detector runs the reference's host loop unchanged.
"""

from __future__ import annotations

import time

import numpy as np

from ..solution.snapshot import SnapshotWriter
from .solver_base import Solver


# Consecutive detections without pairs after which the device loop steps speculatively
# (detection beside the step, the step discarded if pairs turn up): a discarded step costs a
# whole step, the overlap saves about the detection's time, so it pays only when merges are rare.
SPECULATE_AFTER = 8


class EulerDropletSolver(Solver):
    def __init__(self, force_calculator, solution, post_processor, collision_detector=None, save_interval: int = 1,
                 pbm_coupling=None, verbose: bool = True, snapshot_depth: int = 4, graphs: bool = True):
        self.force_calculator = force_calculator
        self.solution = solution
        self.post_processor = post_processor
        self.collision_detector = collision_detector
        self.pbm_coupling = pbm_coupling
        self.simulation_time = 0
        self.save_interval = max(save_interval, 1)
        self.verbose = verbose
        eta_oil = self.force_calculator.eta_oil
        eta_water = self.force_calculator.eta_water
        self.stokes_factor = 2 * np.pi * eta_oil * (2 * eta_oil + 3 * eta_water) / (eta_oil + eta_water)  # :39-41
        self.steps_taken = 0
        self.snapshot_depth = snapshot_depth  # frames in flight on the device path (0: copy synchronously)
        self.graphs = graphs  # replay the direct step as a CUDA graph (device path, direct calculator)
        self.graph_replays = 0

    # ------------------------------------------------------------------
    def _device_capable(self) -> bool:
        fc, det = self.force_calculator, self.collision_detector
        fc_ok = hasattr(fc, "forces_and_convection_soa") or hasattr(fc, "forces_and_total_velocity_soa")
        det_ok = det is None or hasattr(det, "detect_device")
        return fc_ok and det_ok

    def _progress(self, t, t_start, t_end, time_start, last_percent):
        percent = int(100 * (t - t_start) / max(t_end - t_start, 1e-12))
        if percent != last_percent:
            if self.verbose:
                print(f"{percent}%: time {t:.3f} of {t_end:.3f}, droplets: {self.solution.num_particles}, "
                      f"elapsed: {time.time() - time_start:.1f} s", flush=True)
        return percent

    def solve(self, dt, total_time):
        if self._device_capable():
            self._solve_device(dt, total_time)
        else:
            self._solve_host(dt, total_time)

    # ------------------------------------------------------------------
    # reference host loop (euler_droplet_solver.py:43-159), any duck-typed parts
    # ------------------------------------------------------------------
    def _solve_host(self, dt, total_time):
        t = float(self.solution.get_current_time())
        t_start = t
        t_end = t_start + float(total_time)
        is_aborted = False
        time_start = time.time()
        last_percent = -1
        while (t < t_end) and not is_aborted:
            if self.post_processor.stop_simulation:
                break
            positions = self.solution.initial_droplet_state.positions
            radii = self.solution.initial_droplet_state.radii
            remaining_steps = int((t_end - t) / dt) + 1
            for step in range(remaining_steps):
                last_percent = self._progress(t, t_start, t_end, time_start, last_percent)
                if self.post_processor.stop_simulation:
                    is_aborted = True
                    break
                if self.collision_detector is not None:
                    is_collision, collided_pairs = self.collision_detector.detect(positions, radii)
                    if is_collision:
                        if self.pbm_coupling is not None:
                            self.pbm_coupling.on_collision(collided_pairs, radii)
                        self.solution.is_collision = True
                        self.solution.collided_droplets = collided_pairs
                        self.solution.compact()
                        self.solution = self.solution.generate_next_solution()
                        self.post_processor.update_solution(self.solution)
                        if self.solution.real_time_visualization:
                            self.post_processor.update_live_plot()
                        break
                if hasattr(self.force_calculator, "calculate_forces_and_total_velocity"):
                    _, total_velocities = self.force_calculator.calculate_forces_and_total_velocity(
                        positions, radii, stokes_factor=self.stokes_factor)
                    positions += total_velocities * dt
                else:
                    forces, convection_velocities = self.force_calculator.calculate_forces_and_convection(
                        positions, radii)
                    migration_velocities = forces / (self.stokes_factor * radii[:, np.newaxis])
                    positions += (migration_velocities + convection_velocities) * dt
                if self.force_calculator.boundary_mode == "periodic":
                    positions %= self.force_calculator.L
                if self.pbm_coupling is not None:
                    self.pbm_coupling.step(t + dt, radii, dt)
                t += dt
                self.steps_taken += 1
                if self.save_interval <= 1 or step % self.save_interval == 0 or step == remaining_steps - 1:
                    self.solution.save_step(t, positions)
                if self.solution.should_update_visualization():
                    self.post_processor.live_plot()
        self._finish(time_start)

    def _finish(self, time_start):
        self.solution.compact_all()
        self.simulation_time = time.time() - time_start
        if self.verbose:
            print(f"Total computation time: {self.simulation_time:.2f} s")
        if self.solution.real_time_visualization:
            self.post_processor.finalize_live_plot()

    # ------------------------------------------------------------------
    # device-resident loop
    # ------------------------------------------------------------------
    def _solve_device(self, dt, total_time):
        fc, det = self.force_calculator, self.collision_detector
        ctx = fc._ctx
        torch = ctx.torch
        dev = ctx.device
        L = float(fc.L)
        periodic = fc.boundary_mode == "periodic"
        tree = hasattr(fc, "forces_and_total_velocity_soa")

        t = float(self.solution.get_current_time())
        t_start = t
        t_end = t_start + float(total_time)
        is_aborted = False
        time_start = time.time()
        last_percent = -1

        def upload(sol):
            p = np.ascontiguousarray(sol.initial_droplet_state.positions, dtype=np.float64).reshape(-1, 3)
            r = np.ascontiguousarray(sol.initial_droplet_state.radii, dtype=np.float64)
            n = len(r)
            cap = max(n, 1)
            bufs = [torch.empty((3, cap), dtype=torch.float64, device=dev) for _ in range(2)]
            rb = [torch.empty(cap, dtype=torch.float64, device=dev) for _ in range(2)]
            aos = torch.as_tensor(p, device=dev)
            if n:
                ctx.aos_to_soa(n, aos, bufs[0])
                rb[0][:n].copy_(torch.as_tensor(r, device=dev))
            return n, bufs, rb

        n, pos_bufs, r_bufs = upload(self.solution)
        cur = 0  # positions double buffer
        rc = 0  # radii buffer (changes only on a merge)
        host_frame = torch.empty((max(n, 1), 3), dtype=torch.float64, pin_memory=True)
        aos_dev = torch.empty((max(n, 1), 3), dtype=torch.float64, device=dev)
        n_out = torch.zeros(1, dtype=torch.int32, device=dev)
        radii_host = np.ascontiguousarray(self.solution.initial_droplet_state.radii, dtype=np.float64)

        def frame(nn):
            ctx.soa_to_aos(nn, pos_bufs[cur], aos_dev)
            host_frame[:nn].copy_(aos_dev[:nn], non_blocking=True)
            torch.cuda.current_stream(dev).synchronize()
            return host_frame[:nn].numpy()

        writer = SnapshotWriter(ctx, n, self.snapshot_depth) if self.snapshot_depth > 0 else None

        from .. import _native as N

        state = {"graphs": self.graphs and not tree}
        graphs = {}  # (n, cur, rc, detect) -> (graph, kernels in it); a key is captured on its second use
        seen = set()
        speculative = det is not None and hasattr(det, "detect_launch") and hasattr(det, "_pairs")
        side = torch.cuda.Stream(device=dev)  # the speculative step's detection
        clean = [0]  # consecutive detections without pairs
        pairs_ptr = [det._pairs.data_ptr() if speculative else 0]

        def advance(n, cur, rc, detect=False):
            """[detection of pos_bufs[cur] +] forces + convection + Euler from pos_bufs[cur]
            into pos_bufs[1 - cur]."""
            def body():
                main = torch.cuda.current_stream(dev)
                if detect:  # on a side stream, beside the step
                    side.wait_stream(main)
                    with torch.cuda.stream(side):
                        det.detect_launch(n, pos_bufs[cur], r_bufs[rc], L, periodic)
                F, V = fc.forces_and_convection_soa(n, pos_bufs[cur], r_bufs[rc])
                ctx.euler_update(n, pos_bufs[cur], r_bufs[rc], F, V, self.stokes_factor, dt, L, periodic,
                                 pos_bufs[1 - cur])
                if detect:
                    main.wait_stream(side)

            key = (n, cur, rc, detect)
            if not state["graphs"] or key not in seen:
                seen.add(key)  # the first call runs eagerly: it sizes every buffer the capture reuses
                body()
                return
            if key not in graphs:
                g = torch.cuda.CUDAGraph()
                c0 = N.launch_count()
                try:
                    with torch.cuda.graph(g, capture_error_mode="thread_local"):
                        body()
                except RuntimeError as e:  # a calculator whose calls cannot be captured: run eagerly
                    state["graphs"] = False
                    if self.verbose:
                        print(f"CUDA graph capture unavailable ({e}); stepping without graphs")
                    body()
                    return
                graphs[key] = (g, N.launch_count() - c0)
            g, k = graphs[key]
            g.replay()
            N.count_replayed_launches(k)
            self.graph_replays += 1

        def save(tt, nn):
            if writer is None:
                self.solution.save_step(tt, frame(nn))
            else:
                writer.push(self.solution, tt, pos_bufs[cur], nn)

        while (t < t_end) and not is_aborted:
            if self.post_processor.stop_simulation:
                break
            remaining_steps = int((t_end - t) / dt) + 1
            for step in range(remaining_steps):
                last_percent = self._progress(t, t_start, t_end, time_start, last_percent)
                if self.post_processor.stop_simulation:
                    is_aborted = True
                    break
                pos, r = pos_bufs[cur], r_bufs[rc]
                stepped = False
                if det is not None and n > 0:
                    # a speculative step is discarded when pairs are found, so it pays only while
                    # collisions are rare: after SPECULATE_AFTER consecutive detections without pairs
                    if tree or not speculative or clean[0] < SPECULATE_AFTER:
                        k, pairs, counts = det.detect_device(n, pos, r, L, periodic)
                    else:  # detection and the step together; the step is kept when no pair was found
                        advance(n, cur, rc, detect=True)
                        torch.cuda.current_stream(dev).synchronize()
                        k, pairs, counts = det.detect_finish(n, pos, r, L, periodic)
                        if det._pairs.data_ptr() != pairs_ptr[0]:  # the pair buffer grew: recapture
                            pairs_ptr[0] = det._pairs.data_ptr()
                            graphs.clear()
                            seen.clear()
                        stepped = k == 0
                    clean[0] = clean[0] + 1 if k == 0 else 0
                    if k > 0:
                        if writer is not None:
                            writer.flush()  # this solution's frames first
                        pairs_host = pairs.cpu().numpy()
                        if self.pbm_coupling is not None:
                            self.pbm_coupling.on_collision(pairs_host, radii_host)
                        self.solution.is_collision = True
                        self.solution.collided_droplets = pairs_host
                        self.solution.compact()
                        nxt = 1 - cur
                        ctx.merge(n, pos, r, pairs, counts, pos_bufs[nxt], r_bufs[1 - rc], n_out)
                        n = int(n_out.item())
                        graphs.clear()  # captured for the old droplet count
                        seen.clear()
                        cur, rc = nxt, 1 - rc
                        new_pos = frame(n).copy()
                        radii_host = r_bufs[rc][:n].cpu().numpy()
                        self.solution.initial_droplet_state.positions[...] = self.solution.get_current_positions()
                        self.solution = self.solution._next_from_state(new_pos, radii_host)
                        self.post_processor.update_solution(self.solution)
                        if self.solution.real_time_visualization:
                            self.post_processor.update_live_plot()
                        break
                nxt = 1 - cur
                if n > 0 and not stepped:
                    if tree:
                        V = fc.forces_and_total_velocity_soa(n, pos, r, self.stokes_factor)
                        ctx.euler_update_total(n, pos, V, dt, L, periodic, pos_bufs[nxt])
                    else:
                        advance(n, cur, rc)
                cur = nxt
                if self.pbm_coupling is not None:
                    self.pbm_coupling.step(t + dt, radii_host, dt)
                t += dt
                self.steps_taken += 1
                if self.save_interval <= 1 or step % self.save_interval == 0 or step == remaining_steps - 1:
                    save(t, n)
                if self.solution.should_update_visualization():
                    if writer is not None:
                        writer.flush()
                    self.post_processor.live_plot()
        if writer is not None:
            writer.flush()
        # the reference integrates in place into initial_droplet_state.positions
        if n > 0:
            self.solution.initial_droplet_state.positions[...] = frame(n)
        ctx.raise_device_errors()
        self._finish(time_start)
