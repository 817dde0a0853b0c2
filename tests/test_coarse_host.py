"""Host logic of the two-level preconditioner, on the CPU.

* The balanced aggregation (csrc/octree.h, the library's own host code,
  built by oracle/Makefile into lib/liboctree_shim.so): every member gets a
  box; the boxes are disjoint axis-aligned cell boxes; the count stays within
  the limit and comes within seven of it while a box can still split; boxes
  are finer where the records are denser; the result depends on the input
  only.
* The blocked in-place Gauss-Jordan of coarse_build, restated in NumPy
  (oracle/gauss_jordan.py) with the same panel sweeps, deferred row
  interchanges, rank-`panel` updates and column order: equal to
  numpy.linalg.inv on non-symmetric matrices that need pivoting, with a last
  panel narrower than the others.
"""
import ctypes
import os

import numpy as np
import pytest

import gauss_jordan

HERE = os.path.dirname(os.path.abspath(__file__))
SHIM = os.path.join(HERE, "..", "oracle", "lib", "liboctree_shim.so")

needs_shim = pytest.mark.skipif(not os.path.exists(SHIM), reason="oracle/lib/liboctree_shim.so not built (make -C oracle)")


def _aggregate(cell, B, NI, NJ, NK, maxagg):
    L = ctypes.CDLL(SHIM)
    L.octree_aggregates_c.restype = ctypes.c_int
    cell = np.ascontiguousarray(cell, dtype=np.int32)
    n = len(cell) // 3
    box = np.full(n, -1, dtype=np.int32)
    rc = L.octree_aggregates_c(cell.ctypes.data_as(ctypes.c_void_p), n, B, NI, NJ, NK, maxagg,
                               box.ctypes.data_as(ctypes.c_void_p))
    assert rc == 0
    return box


def _refined_cells(NI=48, NJ=24, NK=12, seed=3):
    # eight records per cell, 64 in a refined block (as APR children pack them)
    rng = np.random.default_rng(seed)
    cells = []
    for z in range(NK):
        for y in range(NJ):
            for x in range(NI):
                per = 64 if (10 <= x < 22 and 6 <= y < 16 and z < 6) else 8
                cells += [(x, y, z)] * per
    cells = np.array(cells, dtype=np.int32)
    return cells[rng.permutation(len(cells))].reshape(-1), NI, NJ, NK


@needs_shim
@pytest.mark.parametrize("maxagg", [64, 500, 2000])
def test_balanced_aggregates_are_disjoint_boxes_within_the_limit(maxagg):
    cell, NI, NJ, NK = _refined_cells()
    box = _aggregate(cell, 16, NI, NJ, NK, maxagg)
    c = cell.reshape(-1, 3)
    assert (box >= 0).all()
    m = int(box.max()) + 1
    assert m <= maxagg
    ids = np.unique(box)
    assert len(ids) == m                                    # numbered 0 .. m-1
    lo = np.array([c[box == b].min(axis=0) for b in ids])
    hi = np.array([c[box == b].max(axis=0) for b in ids])
    # disjoint: no member of another box inside a box's cell range
    for b in ids:
        inside = np.all((c >= lo[b]) & (c <= hi[b]), axis=1)
        assert (box[inside] == b).all(), b
    # splitting stops at the limit: while a box wider than one cell is left,
    # the next split (up to seven more boxes) would have passed it
    wide = (hi - lo).max(axis=1) > 0
    if wide.any():
        assert m >= maxagg - 7, (m, maxagg)


@needs_shim
def test_balanced_aggregates_follow_the_rows_and_depend_on_the_input_only():
    cell, NI, NJ, NK = _refined_cells()
    a = _aggregate(cell, 16, NI, NJ, NK, 500)
    b = _aggregate(cell, 16, NI, NJ, NK, 500)
    assert np.array_equal(a, b)
    c = cell.reshape(-1, 3)
    refined = (c[:, 0] >= 10) & (c[:, 0] < 22) & (c[:, 1] >= 6) & (c[:, 1] < 16) & (c[:, 2] < 6)
    # finer boxes (fewer cells each) where the records are denser
    cells_per_box = {}
    for bx in np.unique(a):
        sel = a == bx
        cells_per_box[bx] = (len(np.unique(c[sel], axis=0)), bool(refined[sel].all()), bool((~refined[sel]).all()))
    fine = [v[0] for v in cells_per_box.values() if v[1]]
    coarse = [v[0] for v in cells_per_box.values() if v[2]]
    assert fine and coarse and np.median(fine) < np.median(coarse)


@needs_shim
def test_one_cell_boxes_stop_the_splitting():
    # four occupied cells can make at most four boxes, whatever the limit
    cell = np.array([(0, 0, 0)] * 5 + [(1, 0, 0)] * 5 + [(0, 1, 0)] * 5 + [(5, 5, 5)] * 5, dtype=np.int32).reshape(-1)
    box = _aggregate(cell, 8, 8, 8, 8, 100)
    assert int(box.max()) + 1 == 4


@pytest.mark.parametrize("m,panel", [(7, 3), (50, 8), (130, 64), (200, 64)])
def test_blocked_gauss_jordan_equals_the_inverse(m, panel):
    rng = np.random.default_rng(m)
    A = rng.standard_normal((m, m)) + np.diag(rng.uniform(-1.0, 1.0, m))   # needs row interchanges
    X, piv = gauss_jordan.blocked_gauss_jordan(A, panel)
    assert (piv != np.arange(m)).any()
    ref = np.linalg.inv(A)
    assert np.abs(X - ref).max() <= 1e-10 * max(1.0, np.abs(ref).max())
    assert np.abs(A @ X - np.eye(m)).max() <= 1e-10


def test_blocked_gauss_jordan_reports_a_singular_matrix():
    A = np.ones((5, 5))
    with pytest.raises(np.linalg.LinAlgError):
        gauss_jordan.blocked_gauss_jordan(A, 2)
