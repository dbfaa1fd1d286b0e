"""Trajectory frames from the device while the simulation runs on.

The reference appends every saved frame to the solution on the host
(droplet_solution.py:63-92, called from euler_droplet_solver.py:140-144).  On
the device-resident path the positions live in HBM, so a saved frame is a
device-to-host copy.  ``SnapshotWriter`` keeps ``depth`` device staging slots
and pinned host slots: at a save step the positions are converted to (N, 3) in
a device slot on the compute stream, a copy stream waits for that and copies
the slot to its pinned host slot, and the compute stream carries on with the
next steps.  Frames are appended to their solution in order once their copy
has completed -- opportunistically at later saves, and all of them before the
solution chain changes (a merge), before a live plot reads the solution, and at
the end of the run.
"""

from __future__ import annotations

import collections


class SnapshotWriter:
    def __init__(self, ctx, capacity: int, depth: int = 4):
        torch = ctx.torch
        self.ctx = ctx
        self.torch = torch
        self.depth = max(int(depth), 1)
        cap = max(int(capacity), 1)
        dev = ctx.device
        self.dev = [torch.empty((cap, 3), dtype=torch.float64, device=dev) for _ in range(self.depth)]
        self.host = [torch.empty((cap, 3), dtype=torch.float64, pin_memory=True) for _ in range(self.depth)]
        self.ready = [torch.cuda.Event() for _ in range(self.depth)]
        self.done = [torch.cuda.Event() for _ in range(self.depth)]
        self.copy_stream = torch.cuda.Stream(device=dev)
        self.pending = collections.deque()  # (slot, time, n, solution), oldest first
        self.next_slot = 0
        self.frames = 0

    def push(self, solution, t, pos_soa, n: int):
        """Queue the frame (t, positions) of ``solution``; returns at once."""
        while self.pending and self.done[self.pending[0][0]].query():
            self._append_oldest()
        if len(self.pending) == self.depth:  # every slot in flight: wait for the oldest
            self._append_oldest()
        s = self.next_slot
        self.next_slot = (s + 1) % self.depth
        compute = self.torch.cuda.current_stream(self.ctx.device)
        if n > 0:
            self.ctx.soa_to_aos(n, pos_soa, self.dev[s])
        self.ready[s].record(compute)
        with self.torch.cuda.stream(self.copy_stream):
            self.copy_stream.wait_event(self.ready[s])
            if n > 0:
                self.host[s][:n].copy_(self.dev[s][:n], non_blocking=True)
            self.done[s].record(self.copy_stream)
        self.dev[s].record_stream(self.copy_stream)  # the allocator must not hand the slot out while it is read
        self.pending.append((s, t, n, solution))

    def _append_oldest(self):
        s, t, n, sol = self.pending.popleft()
        self.done[s].synchronize()
        sol.save_step(t, self.host[s][:n].numpy())
        self.frames += 1

    def flush(self):
        """Append every queued frame (blocks until their copies are done)."""
        while self.pending:
            self._append_oldest()
