"""Collision counts between volume classes (pbm/collision_frequency of the
reference) on the GPU, against the reference's own outputs
(tests/golden/collfreq_*.npz): the tree walk over the FP64 flat octree
(csrc/tree.cu) and the hash-pair form (csrc/hash.cu) bit-exact, the volume
classes identical."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

CASES = sorted(p.name for p in GOLDEN.glob("collfreq_*.npz"))


def _grid(g):
    from pbm import VolumeGrid

    return VolumeGrid.from_radii_range(float(g["r_min"]), float(g["r_max"]), int(g["n_bins"]), str(g["spacing"]))


@pytest.mark.parametrize("name", CASES)
def test_tree_and_direct_matrices_bit_exact(golden, name):
    from dem.octree import FlatOctree
    from pbm.collision_frequency import DirectCollisionFrequency, TreeCollisionFrequency

    g = golden(name)
    pos, r, L, per = g["positions"], g["radii"], float(g["L"]), bool(g["periodic"])
    grid = _grid(g)
    np.testing.assert_array_equal(grid.edges, g["edges"])
    np.testing.assert_array_equal(grid.bin_indices((4.0 / 3.0) * np.pi * r**3), g["bins"])
    n = len(r)
    tree = FlatOctree(theta=0.5, mpl=int(g["mpl"]), num_particles=n)
    tree.build(pos, r, L, per)
    M = TreeCollisionFrequency(tree, grid, max_particles=n).compute(pos, r)
    np.testing.assert_array_equal(M, g["matrix_tree"])
    np.testing.assert_array_equal(M, M.T)
    D = DirectCollisionFrequency(grid).compute(pos, r, L=L, periodic=per)
    np.testing.assert_array_equal(D, g["matrix_direct"])
    assert tree._ctx.device_errors() == 0


def test_direct_matches_detector_pairs_at_scale():
    """N = 20,000 touching droplets: the matrix sums to twice the detector's pair count."""
    from dem.collision_detector import SpatialHashCollisionDetector
    from pbm import VolumeGrid
    from pbm.collision_frequency import DirectCollisionFrequency

    rng = np.random.default_rng(5)
    n, L = 20000, 2e-3
    pos = rng.uniform(0, L, (n, 3))
    r = rng.uniform(5e-6, 30e-6, n)
    grid = VolumeGrid.from_radii_range(5e-6, 30e-6, 8)
    D = DirectCollisionFrequency(grid).compute(pos, r, L=L, periodic=True)
    hit, pairs = SpatialHashCollisionDetector(num_particles=n, L=L).detect(pos, r)
    assert hit and D.sum() == 2 * len(pairs)
    b = grid.bin_indices((4.0 / 3.0) * np.pi * r**3)
    ref = np.zeros_like(D)
    np.add.at(ref, (b[pairs[:, 0]], b[pairs[:, 1]]), 1)
    np.add.at(ref, (b[pairs[:, 1]], b[pairs[:, 0]]), 1)
    np.testing.assert_array_equal(D, ref)
