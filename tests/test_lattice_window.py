"""The host-side lattice window of the sync-free remesh (no GPU): the window
computed from the blobs' bounding box holds exactly the range of the
reference's left indices (oracle restatement of ``_regridding.py:157``),
including blobs on cell boundaries."""
import numpy as np
import pytest

import oracle
from pfblob.regrid import lattice_window


@pytest.mark.parametrize("seed", range(6))
def test_window_equals_the_range_of_left_indices(seed):
    rng = np.random.default_rng(seed)
    h = float(rng.uniform(1e-4, 0.05))
    xb0 = yb0 = -1.5 * h
    n = 5000
    cx, cy = rng.uniform(-3, 3, 2)
    x = cx + rng.uniform(-0.5, 0.5, n)
    y = cy + rng.uniform(-0.2, 0.7, n)
    # blobs exactly on lattice nodes and on cell edges
    k = rng.integers(-2000, 2000, 200)
    x[:200] = k * h + 0.5 * h + xb0
    y[200:400] = k * h + xb0
    lx = oracle.remesh_left_index(x, xb0, h)
    ly = oracle.remesh_left_index(y, yb0, h)
    box = (x.min(), x.max(), y.min(), y.max())
    ixmin, iymin, nbx, nby = lattice_window(box, h, xb0, yb0)
    assert (ixmin, iymin) == (lx.min(), ly.min())
    assert (ixmin + nbx - 1, iymin + nby - 1) == (lx.max(), ly.max())


def test_single_point_window():
    h = 0.01
    ixmin, iymin, nbx, nby = lattice_window((0.3, 0.3, 0.7, 0.7), h, -1.5 * h, -1.5 * h)
    assert (nbx, nby) == (1, 1)
    assert ixmin == oracle.remesh_left_index(np.array([0.3]), -1.5 * h, h)[0]
    assert iymin == oracle.remesh_left_index(np.array([0.7]), -1.5 * h, h)[0]
