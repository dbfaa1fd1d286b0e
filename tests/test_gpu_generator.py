"""The device droplet generator (csrc/gen.cu, dem.particle_generator.
UniformDropletGenerator): the reference's rejection rule
(uniform_droplet_generator.py:107-164) checked on its outputs -- no two
droplets closer than r_i + r_j + minimum_distance (plain distance, or the
minimum image when periodic), radii and positions in range, the same seed
giving the same state, ValueError when the droplets cannot be placed."""

from __future__ import annotations

import numpy as np
import pytest
from scipy.spatial import cKDTree

pytestmark = pytest.mark.gpu


def _gen(**kw):
    from dem.particle_generator import UniformDropletGenerator

    g = UniformDropletGenerator(**kw)
    return g, g.generate()


def _min_clearance(pos, r, gap, L=None):
    """min over pairs of d - (r_i + r_j + gap), from every pair within reach."""
    tree = cKDTree(np.mod(pos, L), boxsize=L) if L else cKDTree(pos)
    pairs = tree.query_pairs(2 * r.max() + gap + 1e-12, output_type="ndarray")
    if len(pairs) == 0:
        return np.inf
    d = pos[pairs[:, 1]] - pos[pairs[:, 0]]
    if L:
        d -= L * np.rint(d / L)
    return float((np.sqrt((d * d).sum(1)) - (r[pairs[:, 0]] + r[pairs[:, 1]] + gap)).min())


@pytest.mark.parametrize("periodic", [False, True])
def test_no_overlaps_and_ranges(periodic):
    lo, hi, gap = 0.2e-3, 1.2e-3, 1e-6
    g, st = _gen(coord_range=(lo, hi), radii_range=(5e-6, 20e-6), num_particles=6000, minimum_distance=gap, seed=3,
                 periodic=periodic)
    pos, r = st.positions, st.radii
    assert pos.shape == (6000, 3) and r.shape == (6000,)
    assert pos.min() >= lo and pos.max() < hi and r.min() >= 5e-6 and r.max() <= 20e-6
    assert g.rounds > 1  # the first draw overlaps at this density
    L = (hi - lo) if periodic else None
    assert _min_clearance(pos - lo, r, gap, L) > -1e-15
    # uniform: mean near the middle, every octant populated
    assert abs(pos.mean() - 0.5 * (lo + hi)) < 0.02 * (hi - lo)
    assert abs(r.mean() - 12.5e-6) < 0.5e-6


def test_seed_fixes_the_state():
    kw = dict(coord_range=(0.0, 1e-3), radii_range=(5e-6, 20e-6), num_particles=3000, minimum_distance=1e-6)
    _, a = _gen(seed=11, **kw)
    _, b = _gen(seed=11, **kw)
    _, c = _gen(seed=12, **kw)
    np.testing.assert_array_equal(a.positions, b.positions)
    np.testing.assert_array_equal(a.radii, b.radii)
    assert not np.array_equal(a.positions, c.positions)


def test_impossible_packing_raises_and_edge_sizes():
    with pytest.raises(ValueError):
        _gen(coord_range=(0.0, 1.0), radii_range=(0.3, 0.3), num_particles=40, seed=1, max_rounds=30)
    _, st = _gen(coord_range=(0.0, 1.0), radii_range=(0.01, 0.02), num_particles=0, seed=1)
    assert st.positions.shape == (0, 3) and len(st.radii) == 0
    _, st = _gen(coord_range=(0.0, 1.0), radii_range=(0.01, 0.02), num_particles=1, seed=1)
    assert st.positions.shape == (1, 3)


@pytest.mark.parametrize("n,seed,periodic,gap", [(2000, 0, True, 1e-6), (3000, 7, False, 1e-6),
                                                 (65536, 0, True, 1e-6), (4096, 0, True, -2e-6)])
def test_lognormal_generator_device_search_gives_the_host_state(n, seed, periodic, gap):
    """The seeded lognormal states of the measured configurations are the same
    whether the overlap rounds search on the GPU (whole-cell hash) or on the
    host (scipy cKDTree)."""
    from dem.particle_generator import LognormalDropletGenerator

    a = LognormalDropletGenerator(n, seed=seed, periodic=periodic, minimum_distance=gap, device="host")
    b = LognormalDropletGenerator(n, seed=seed, periodic=periodic, minimum_distance=gap, device="auto")
    sa, sb = a.generate(), b.generate()
    assert a.L == b.L
    np.testing.assert_array_equal(sa.radii, sb.radii)
    np.testing.assert_array_equal(sa.positions, sb.positions)
