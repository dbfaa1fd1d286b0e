"""pbm.VolumeGrid (host) against the reference's classes in the golden cases."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import GOLDEN


@pytest.mark.parametrize("name", sorted(p.name for p in GOLDEN.glob("collfreq_*.npz")))
def test_edges_and_bins(golden, name):
    from pbm import VolumeGrid

    g = golden(name)
    grid = VolumeGrid.from_radii_range(float(g["r_min"]), float(g["r_max"]), int(g["n_bins"]), str(g["spacing"]))
    np.testing.assert_array_equal(grid.edges, g["edges"])
    np.testing.assert_array_equal(grid.bin_indices((4.0 / 3.0) * np.pi * g["radii"] ** 3), g["bins"])


def test_errors_and_clamping():
    from pbm import VolumeGrid

    with pytest.raises(ValueError):
        VolumeGrid(0.0, 1.0, 4)
    with pytest.raises(ValueError):
        VolumeGrid(1.0, 2.0, 1)
    with pytest.raises(ValueError):
        VolumeGrid(1.0, 2.0, 4, spacing="cubic")
    g = VolumeGrid(1.0, 16.0, 4)
    np.testing.assert_allclose(g.edges, [1.0, 2.0, 4.0, 8.0, 16.0], rtol=1e-14)
    assert [g.bin_index(v) for v in (0.5, 1.0, 3.9, 16.0, 99.0)] == [0, 0, 1, 3, 3]
    np.testing.assert_array_equal(g.bin_indices(np.array([0.5, 2.5, 8.5, 99.0])), [0, 1, 3, 3])
