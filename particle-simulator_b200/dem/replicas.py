"""Multi-GPU runs as independent replicas.

The droplet step has no exchange between boxes: on N GPUs (one process per
GPU, ``torch.distributed`` for the plumbing) every rank integrates its own
seeded box and no data moves between ranks.  The job's time for K steps is the
slowest rank's, and its throughput is the units all ranks processed over that
time (weak scaling).  These helpers are the whole of that logic.
"""

from __future__ import annotations


def replica_seed(seed: int, rank: int) -> int:
    """Rank r integrates the box drawn with seed + r."""
    return int(seed) + int(rank)


def job_time_ms(local_ms: float, device=None) -> float:
    """The slowest rank's time (all-reduce MAX over the default process group;
    the local time when there is no group or one rank)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(local_ms)
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, world: int, job_ms: float) -> float:
    """Units of all ranks per second of the slowest rank."""
    return float(units_per_rank) * int(world) / (float(job_ms) / 1000.0)
