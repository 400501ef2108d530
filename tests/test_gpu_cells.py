"""Bit-exact cell binning: the GPU cell build must equal the oracle's project
binning (integer cells, stable order by original index) for the same input."""
import numpy as np
import pytest

import md_simulation_cuda_b200 as mdb
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def _check(pos, Lx, Ly, cell_min):
    cell, perm, ncx, ncy = mdb.cell_build(pos, Lx, Ly, cell_min)
    c2, p2, nx2, ny2 = po.cell_build(pos, Lx, Ly, cell_min)
    assert (ncx, ncy) == (nx2, ny2)
    assert np.array_equal(cell, c2)
    assert np.array_equal(perm, p2)


@pytest.mark.parametrize("n,Lx,Ly,cm,seed", [
    (1000, 50.0, 30.0, 2.8, 0),
    (20000, 141.42, 141.42, 2.8, 1),
    (4096, 71.554, 71.554, 2.8, 2),
    (3000, 12.0, 200.0, 2.5, 3),
    (50, 8.0, 8.0, 2.8, 4),   # a 2x2 grid
])
def test_binning_bit_exact(built, n, Lx, Ly, cm, seed):
    rng = np.random.default_rng(seed)
    pos = np.stack([rng.uniform(0, Lx, n), rng.uniform(0, Ly, n)], axis=1)
    _check(pos, Lx, Ly, cm)


def test_binning_edges(built):
    """x == L after a wrap, values on cell boundaries, negatives and values
    past the box (clamped), and duplicated positions (order kept)."""
    Lx, Ly, cm = 30.0, 21.0, 2.9
    ncx, ncy = int(np.floor(Lx / cm)), int(np.floor(Ly / cm))
    wx, wy = Lx / ncx, Ly / ncy
    pts = [[0.0, 0.0], [Lx, Ly], [Lx, 0.0], [wx, wy], [2 * wx, 3 * wy],
           [np.nextafter(wx, 0), np.nextafter(wy, 0)], [-1e-12, 5.0], [5.0, -3.0],
           [Lx + 4.0, Ly + 9.0], [7.0, 7.0], [7.0, 7.0], [7.0, 7.0]]
    rng = np.random.default_rng(5)
    pos = np.concatenate([np.array(pts), rng.uniform(0, Lx, (500, 2)) * [1, Ly / Lx]])
    _check(pos, Lx, Ly, cm)


def test_binning_deterministic(built):
    rng = np.random.default_rng(6)
    pos = rng.uniform(0, 100, (30000, 2))
    a = mdb.cell_build(pos, 100.0, 100.0, 2.8)
    b = mdb.cell_build(pos, 100.0, 100.0, 2.8)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
