"""The multi-GPU path of bench.py (independent replicas, no collective on the
data path) on CPU: two gloo ranks, each with its own seeded box; the job time is
the slowest rank's and the rate counts every rank's units."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import PKG


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys

    sys.path.insert(0, str(PKG))
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from dem.particle_generator import LognormalDropletGenerator
        from dem.replicas import job_time_ms, replica_seed, whole_job_rate

        g = LognormalDropletGenerator(300, seed=replica_seed(0, rank), device="host")
        st = g.generate()
        local_ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        job = job_time_ms(local_ms)
        out.put((rank, float(st.positions[0, 0]), job, whole_job_rate(20, world, job)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=10) for _ in range(2))
    (r0, x0, job0, rate0), (r1, x1, job1, rate1) = res
    assert x0 != x1  # different seeded boxes
    assert job0 == job1 == 15.0  # max over ranks
    assert rate0 == rate1 == pytest.approx(20 * 2 / 0.015)


def test_single_process_helpers():
    import sys

    sys.path.insert(0, str(PKG))
    from dem.replicas import job_time_ms, replica_seed, whole_job_rate

    assert replica_seed(5, 3) == 8
    assert job_time_ms(12.5) == 12.5  # no process group
    assert whole_job_rate(10, 1, 1000.0) == pytest.approx(10.0)
    assert np.isfinite(whole_job_rate(1, 8, 0.5))
