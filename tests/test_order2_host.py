"""Host logic of the Order2 GPU path, checked without a GPU: the edge-basis order the library
derives from the cells' global vertex ids is the reference's edge numbering as the restatement
(oracle/order2.py, pinned against the reference's topology) orders it."""
import numpy as np
import pytest

from multiscalefemsolver3d_b200 import cells as gcells
from oracle import order2 as o2


def _edge_info(e):
    axis, s, t = e // 4, (e >> 1) & 1, e & 1
    o0, o1 = (1 if axis == 0 else 0), (1 if axis == 2 else 2)
    vl = (s << o0) | (t << o1)
    return vl, vl | (1 << axis)


def test_order2_edge_order_matches_restatement(lib):
    rng = np.random.default_rng(0)
    cv = np.array([rng.permutation(50)[:8] for _ in range(40)], np.int32)
    _, cv_grid, _ = o2.graded_cells(2, 1, 0.0)
    cv = np.concatenate([cv, cv_grid.astype(np.int32)])
    got = gcells.order2_edge_order(cv)
    for c in range(cv.shape[0]):
        topo = o2._Topo(cv[c])
        for k, e in enumerate(got[c]):
            vl, vh = _edge_info(int(e))
            assert set(topo.edges[k]) == {vl, vh}


def test_order2_edge_order_rejects_repeated_vertices(lib):
    with pytest.raises(Exception):
        gcells.order2_edge_order(np.array([[0, 1, 2, 3, 4, 5, 6, 6]], np.int32))
