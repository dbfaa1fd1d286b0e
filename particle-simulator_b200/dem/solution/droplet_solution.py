"""Trajectory buffer and chain of solutions split at coalescence events.

Drop-in for dem/solution/droplet_solution.py:10-499 of
ddkx21/particle-simulator (same attributes, methods and ``.npz`` chain
format).  The coalescence step of ``generate_next_solution`` (:208-287) runs
in the merge kernel of libdem_b200 (csrc/merge.cu).
"""

from __future__ import annotations

import os.path
import threading
import time

import numpy as np

from ..particle_state import DropletState
from .solution_base import Solution

_merge_ctx = {}
_merge_lock = threading.Lock()


def _merge_context(capacity: int):
    from .. import _native as N
    from .._io import Stager

    torch = N._torch()
    dev = torch.cuda.current_device()
    with _merge_lock:
        entry = _merge_ctx.get(dev)
        if entry is None:
            ctx = N.Context(max(capacity, 1), dev)
            entry = (ctx, Stager(ctx))
            _merge_ctx[dev] = entry
        ctx, io = entry
        if capacity > ctx.capacity:
            ctx.reserve(capacity)
    return entry


def order_pairs(pairs) -> np.ndarray:
    """Collision pairs ordered by their first index (stable), as
    droplet_solution.py:229-230 orders them."""
    pairs = np.asarray(pairs, dtype=np.int32).reshape(-1, 2)
    return pairs[np.argsort(pairs[:, 0], kind="stable")]


def merge_droplets(positions: np.ndarray, radii: np.ndarray, pairs: np.ndarray):
    """Greedy volume-conserving merge on the device.  Returns (positions, radii)."""
    from .. import _native as N

    pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
    r = np.ascontiguousarray(radii, dtype=np.float64).reshape(-1)
    n = len(r)
    ctx, io = _merge_context(n)
    torch = ctx.torch
    st, _ = io.positions(pos, r, tag="merge")
    pairs = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
    if len(pairs) and (pairs.min() < 0 or pairs.max() >= n):
        raise IndexError("collision pair index out of range")
    dpairs = torch.as_tensor(pairs.copy(), device=ctx.device) if len(pairs) else torch.zeros(
        (1, 2), dtype=torch.int32, device=ctx.device)
    k = torch.tensor([len(pairs)], dtype=torch.int64, device=ctx.device)
    out_pos = io.buf.dev("merge_out_pos", (3, n))
    out_r = torch.empty(n, dtype=torch.float64, device=ctx.device)
    n_out = torch.zeros(1, dtype=torch.int32, device=ctx.device)
    ctx.merge(n, st.pos, st.r, dpairs, k, out_pos, out_r, n_out)
    m = int(n_out.item())
    p_new, = io.download([out_pos[:, :m]], m) if m else (np.zeros((0, 3)),)
    r_new = out_r[:m].cpu().numpy()
    ctx.raise_device_errors()
    return p_new, r_new


class DropletSolution(Solution):
    def __init__(
        self,
        initial_droplet_state,
        real_time_visualization=False,
        update_interval=0.05,
        length=10,
        previous=None,
        filename=None,
    ):
        self.initial_droplet_state = initial_droplet_state
        self.num_particles = len(initial_droplet_state.radii)
        self.radii = initial_droplet_state.radii
        self.length = length
        self.real_time_visualization = real_time_visualization
        self.update_interval = update_interval
        self.times = np.zeros((self.length, 1)) + initial_droplet_state.time
        self.trajectories = np.zeros((self.length, self.num_particles, 3))
        self.last_update_time = time.time()
        self._prev = previous
        self._next = None
        self.is_collision = False
        self.collided_droplets = []
        self.resulting_droplet = []
        self.current_step = -1
        self.save_step(initial_droplet_state.time, initial_droplet_state.positions)
        self.filename = filename

    def save_step(self, t, positions):
        """droplet_solution.py:63-92 (buffers double when full)."""
        self.current_step += 1
        if self.current_step >= self.length:
            new_length = self.length * 2
            new_times = np.empty((new_length, 1), dtype=self.times.dtype)
            new_times[: self.length] = self.times
            self.times = new_times
            new_traj = np.empty((new_length, self.num_particles, 3), dtype=self.trajectories.dtype)
            new_traj[: self.length] = self.trajectories
            self.trajectories = new_traj
            self.length = new_length
        self.times[self.current_step] = t
        self.trajectories[self.current_step] = positions

    def get_times(self):
        return self.times[: self.current_step + 1]

    def get_trajectories(self):
        return self.trajectories[: self.current_step + 1]

    def get_current_time(self):
        return self.times[self.current_step][0]

    def get_last_time(self):
        valid_steps = np.where(np.any(self.times != 0, axis=0))[0]
        return self.times[valid_steps[-1]]

    def get_chain_start_time(self):
        return self.get_first_solution().times[0][0]

    def get_chain_end_time(self):
        s = self
        while s._next is not None:
            s = s._next
        return s.times[-1][0]

    def get_first_solution(self):
        s = self
        while s._prev is not None:
            s = s._prev
        return s

    def get_current_positions(self):
        return self.trajectories[self.current_step]

    def compact(self):
        self.times = self.get_times()
        self.trajectories = self.get_trajectories()

    def compact_all(self):
        self.compact()
        s = self._next
        while s is not None:
            s.compact()
            s = s._next
        s = self._prev
        while s is not None:
            s.compact()
            s = s._prev

    def should_update_visualization(self):
        if self.real_time_visualization:
            now = time.time()
            if now - self.last_update_time >= self.update_interval:
                self.last_update_time = now
                return True
        return False

    def _next_from_state(self, new_positions, new_radii):
        new_state = DropletState(new_positions, new_radii, self.times[self.current_step])
        nxt = DropletSolution(
            initial_droplet_state=new_state,
            real_time_visualization=self.real_time_visualization,
            update_interval=self.update_interval,
            length=self.length,
            previous=self,
        )
        self._next = nxt
        nxt.is_collision = False
        return nxt

    def generate_next_solution(self):
        """droplet_solution.py:208-287: merge the colliding droplets on the
        device and chain a new solution that starts at the current time."""
        self.collided_droplets = order_pairs(self.collided_droplets)
        new_positions, new_radii = merge_droplets(self.trajectories[self.current_step], self.radii,
                                                  self.collided_droplets)
        return self._next_from_state(new_positions, new_radii)

    # -- persistence (droplet_solution.py:289-421) -----------------------------
    def save_to_file(self, filename):
        np.savez(filename, num_particles=self.num_particles, radii=self.radii, times=self.get_times(),
                 trajectories=self.get_trajectories())

    def load_from_file(self, filename):
        data = np.load(filename)
        self.num_particles = data["num_particles"]
        self.radii = data["radii"]
        self.times = data["times"]
        self.trajectories = data["trajectories"]
        self.length = len(self.times)
        self.filename = os.path.splitext(os.path.basename(filename))[0]

    def save_chain_to_file(self, filename, precision="float64"):
        dtype = {"float32": np.float32, "float16": np.float16}.get(precision, np.float64)
        s = self.get_first_solution()
        solution_list = []
        while s is not None:
            s.compact()
            solution_list.append(
                {
                    "num_particles": s.num_particles,
                    "radii": s.radii.astype(dtype),
                    "length": s.length,
                    "real_time_visualization": s.real_time_visualization,
                    "update_interval": s.update_interval,
                    "times": s.get_times().astype(dtype),
                    "trajectories": s.get_trajectories().astype(dtype),
                    "is_collision": s.is_collision,
                    "collided_droplets": s.collided_droplets,
                    "resulting_droplet": s.resulting_droplet,
                }
            )
            s = s._next
        np.savez(filename, solutions=solution_list)

    @staticmethod
    def load_chain_from_file(filename):
        fname = os.path.splitext(os.path.basename(filename))[0]
        data = np.load(filename, allow_pickle=True)
        first = prev = None
        for d in data["solutions"]:
            st = DropletState(d["trajectories"][0], d["radii"], d["times"][0])
            s = DropletSolution(
                initial_droplet_state=st,
                real_time_visualization=d["real_time_visualization"],
                update_interval=d["update_interval"],
                length=d["length"],
                previous=prev,
                filename=fname,
            )
            s.times = d["times"]
            s.trajectories = d["trajectories"]
            s.is_collision = d["is_collision"]
            s.collided_droplets = d["collided_droplets"]
            s.resulting_droplet = d["resulting_droplet"]
            if prev is not None:
                prev._next = s
            else:
                first = s
            prev = s
        return first

    def get_state(self, target_time):
        """droplet_solution.py:423-487 (linear interpolation in time)."""
        s = self
        while True:
            tmin, tmax = s.times[0][0], s.times[-1][0]
            if target_time < tmin:
                if s._prev is None:
                    raise ValueError(f"time {target_time} is before the start of the chain")
                s = s._prev
            elif target_time > tmax:
                if s._next is None:
                    raise ValueError(f"time {target_time} is after the end of the chain")
                s = s._next
            else:
                break
        times = s.times.flatten()
        ib = np.searchsorted(times, target_time) - 1
        ia = ib + 1
        ib = max(ib, 0)
        ia = min(ia, len(times) - 1)
        tb, ta = times[ib], times[ia]
        pb, pa = s.trajectories[ib], s.trajectories[ia]
        if target_time == ta:
            p = pa
        elif target_time == tb:
            p = pb
        else:
            p = pb + (target_time - tb) / (ta - tb) * (pa - pb)
        return DropletState(positions=p, radii=s.radii, time=target_time)

    def get_name(self):
        f = self.get_first_solution()
        return f.filename if f.filename is not None else ""
