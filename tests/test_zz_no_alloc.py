"""The allocation-free detector entry point, dem_hash_detect_noalloc.

It serves callers that cannot call cudaMalloc when they detect collisions (a
fixed device-memory budget, a control loop that must not take cudaMalloc's
device-wide synchronisation, an allocator owned by another component).  It
uses a fixed device array inside the library instead of a context workspace.

Checked through the C ABI against the regular entry point, dem_hash_detect,
on two calls in a row with different inputs (the array keeps the previous
call's contents, so the second call also checks that the entry point resets
what must start at zero), at the array's limits (65,536 droplets, 131,072
buckets), in an open box, and with a pair buffer too small for every pair.
Pair sets are integer data: they must be identical.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import dem._native as N

pytestmark = pytest.mark.gpu

MAX_N = 65536
MAX_TABLE = 131072


def _case(n, seed, gap, periodic=True):
    from dem.particle_generator import LognormalDropletGenerator

    g = LognormalDropletGenerator(n, seed=seed, minimum_distance=gap, periodic=periodic)
    s = g.generate()
    return s.positions, s.radii, g.L


def _device_inputs(torch, pos, r):
    soa = torch.as_tensor(np.ascontiguousarray(pos.T), device="cuda")
    return soa, torch.as_tensor(r, device="cuda")


def _via_noalloc(torch, soa, r, L, table, cap, periodic=True):
    n = r.shape[0]
    pairs = torch.full((max(cap, 1), 2), -1, dtype=torch.int32, device="cuda")
    counts = torch.full((2,), -7, dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = N.lib().dem_hash_detect_noalloc(n, soa[0].data_ptr(), soa[1].data_ptr(), soa[2].data_ptr(), r.data_ptr(),
                                          float(L), int(periodic), table, pairs.data_ptr(), cap, counts.data_ptr(),
                                          stream)
    assert rc == N.DEM_OK
    torch.cuda.synchronize()
    k = int(counts[0])
    return k, pairs[: min(k, cap)].cpu().numpy(), int(counts[1])


def _via_context(torch, soa, r, L, table, cap, periodic=True):
    n = r.shape[0]
    ctx = N.Context(n)
    pairs = torch.full((cap, 2), -1, dtype=torch.int32, device="cuda")
    counts = torch.zeros(2, dtype=torch.int64, device="cuda")
    ctx.hash_detect(n, soa, r, L, periodic, table, pairs, cap, counts)
    torch.cuda.synchronize()
    k = int(counts[0])
    assert ctx.device_errors() == 0
    return k, pairs[:k].cpu().numpy(), int(counts[1])


def _table(n):
    table = 1
    while table < 2 * n:
        table <<= 1
    return table


def test_noalloc_matches_context_entry_point_on_two_calls():
    import torch

    # the first call on this device resolves the array's device address; it must not run under stream capture
    assert not torch.cuda.is_current_stream_capturing()
    cases = [(20000, 5, -2e-6), (4096, 6, -1e-6)]  # the second call is smaller than the first
    for n, seed, gap in cases:
        pos, r, L = _case(n, seed, gap)
        soa, rr = _device_inputs(torch, pos, r)
        table = _table(n)
        cap = 4 * n
        got = _via_noalloc(torch, soa, rr, L, table, cap)
        ref = _via_context(torch, soa, rr, L, table, cap)
        assert got[0] == ref[0] and got[0] > 0
        assert got[2] == ref[2]
        np.testing.assert_array_equal(got[1], ref[1])


def test_noalloc_at_its_limits_and_in_an_open_box():
    """n = 65,536 droplets in a table of 131,072 buckets fills every region of
    the array to its last slot; then an open box, where cells clamp at the
    faces instead of wrapping."""
    import torch

    for n, seed, gap, periodic in [(MAX_N, 8, -2e-6, True), (12000, 9, -2e-6, False)]:
        pos, r, L = _case(n, seed, gap, periodic)
        soa, rr = _device_inputs(torch, pos, r)
        table = MAX_TABLE if n == MAX_N else _table(n)
        cap = 4 * n
        got = _via_noalloc(torch, soa, rr, L, table, cap, periodic)
        ref = _via_context(torch, soa, rr, L, table, cap, periodic)
        assert got[0] == ref[0] and got[0] > 0
        assert got[2] == ref[2]
        np.testing.assert_array_equal(got[1], ref[1])


def test_noalloc_overflow_shows_in_the_count_and_keeps_the_first_pairs():
    """With too small a pair buffer the entry point still reports every pair
    in counts[0] (that is the caller's only overflow signal: the error flag
    stays inside the library's array) and writes the lexicographically first
    pair_capacity pairs."""
    import torch

    pos, r, L = _case(6000, 10, -2e-6)
    soa, rr = _device_inputs(torch, pos, r)
    table = _table(6000)
    ref = _via_context(torch, soa, rr, L, table, 4 * 6000)
    assert ref[0] > 40
    for cap in (1, ref[0] // 3, ref[0] - 1):
        got = _via_noalloc(torch, soa, rr, L, table, cap)
        assert got[0] == ref[0] > cap
        np.testing.assert_array_equal(got[1], ref[1][:cap])


def test_noalloc_rejects_sizes_beyond_its_array():
    lib = N.lib()
    null = C.c_void_p(0)
    counts = C.c_void_p(0)
    assert lib.dem_hash_detect_noalloc(MAX_N + 1, null, null, null, null, 1.0, 1, 1024, null, 0, counts, null) == \
        N.DEM_E_CAPACITY
    assert lib.dem_hash_detect_noalloc(100, null, null, null, null, 1.0, 1, 2 * MAX_TABLE, null, 0, counts, null) == \
        N.DEM_E_CAPACITY
    assert lib.dem_hash_detect_noalloc(100, null, null, null, null, 1.0, 1, 1000, null, 0, counts, null) == \
        N.DEM_E_CAPACITY  # not a power of two
