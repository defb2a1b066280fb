"""MsFEM Order2 bases on the GPU (msfem_cells_build_order2) against the restatement
oracle/order2.py, which is pinned against the reference's own Order2 construction
(tests/test_order2_oracle.py)."""
import numpy as np
import pytest

from multiscalefemsolver3d_b200 import cells as gcells
from multiscalefemsolver3d_b200._lib import FP32_IR, FP64
from oracle import order2 as o2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,tol,bound", [(FP64, 1e-11, 1e-8), (FP32_IR, 1e-8, 2e-5)])
def test_order2_bases_match_oracle(lib, cuda, precision, tol, bound):
    """8 graded cells of 4^3 hexahedra with inclusions (E 1:10): every one of the 27 bases of every
    cell within `bound` (relative to the largest value) of the exact restatement, and the 27 x 27
    macro element matrices of those bases within 1e-10 of the restatement's."""
    vxyz, cv, cm = o2.graded_cells(2, 4, 0.5)
    c = gcells.Cells(cm)
    assert c.build_order2(cv, precision, tol) == 0
    got = c.order2_bases()
    K = c.order2_macro_matrices()
    c.close()
    for k in range(cm.n_cells):
        xyz, tets, mat, box = cm.cell(k)
        want = o2.order2_bases(xyz, tets, mat, box, cm.E, cm.nu, cv[k])
        a, b = cm.node_off[k], cm.node_off[k + 1]
        err = np.abs(got[a:b] - want).max() / np.abs(want).max()
        assert err < bound, (k, err)
        if k in (0, 7):
            Kw = o2.macro_element_matrix(xyz, tets, got[a:b], box, cm.E[0], cm.nu[0])
            assert np.abs(K[k] - Kw).max() <= 1e-10 * np.abs(Kw).max()


def test_order2_edge_order_follows_global_vertex_ids(lib, cuda):
    """The same cell with its corners renumbered: the edge bases come back permuted the way the
    ascending (lower, higher) global vertex pairs order them, everything else unchanged."""
    vxyz, cv, cm = o2.graded_cells(1, 4, 0.4)
    g1 = np.arange(8, dtype=np.int32)[None]
    g2 = np.array([[7, 3, 5, 1, 6, 2, 4, 0]], np.int32)
    out = []
    for g in (g1, g2):
        c = gcells.Cells(cm)
        assert c.build_order2(g, FP64, 1e-11) == 0
        out.append(c.order2_bases())
        c.close()
    xyz, tets, mat, box = cm.cell(0)
    for g, got in zip((g1, g2), out):
        want = o2.order2_bases(xyz, tets, mat, box, cm.E, cm.nu, g[0])
        assert np.abs(got - want).max() < 1e-8 * np.abs(want).max()
    np.testing.assert_allclose(out[0][:, :8], out[1][:, :8], atol=1e-8)
    np.testing.assert_allclose(out[0][:, 20:], out[1][:, 20:], atol=1e-8)


@pytest.mark.parametrize("precision,cell_tol,tol,bound", [(FP64, 1e-11, 1e-12, 1e-8), (FP32_IR, 1e-9, 1e-10, 1e-6)])
def test_order2_driver_matches_reference_run(lib, cuda, precision, cell_tol, tol, bound):
    """The composed Order2 driver on the GPU (order2.order2_elastic_driver: GPU bases and element
    matrices, the library's macro CSR, the projected Dirichlet values, GPU Dirichlet rows and
    columns, GPU MINRES) against the reference's own whole Order2 driver run
    (MsFEM::MsFEM_forElasticDeformation_OrderBF2_forPoly, MsFEM/MsFEM.h:14-569, the golden
    fixture tests/golden/msfem_order2.npz made by oracle/_ref's order2_ref --driver): u = 0 on
    z = 0 and (0.01, -0.02, 0.05) on z = 1 over 8 graded cells with inclusions.  FP64 within 1e-8
    relative L2 (the reference's own CG restart loop stops near 1e-9); the FP32 inner solves in
    FP64 refinement within 1e-6."""
    import os

    from multiscalefemsolver3d_b200 import order2 as p2
    d = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "msfem_order2.npz"))
    vxyz, cv, cm = o2.graded_cells(2, 4, 0.5)
    assert abs(cm.xyz.sum() - float(d["xyz_sum_2"])) < 1e-9
    bot = np.nonzero(np.abs(vxyz[:, 2]) < 1e-12)[0]
    top = np.nonzero(np.abs(vxyz[:, 2] - 1) < 1e-12)[0]
    groups = [(bot, (0.0, 0.0, 0.0), (1, 1, 1)), (top, (0.01, -0.02, 0.05), (1, 1, 1))]
    x, info = p2.order2_elastic_driver(cm, vxyz, cv, groups, precision=precision, tol=tol, cell_tol=cell_tol)
    assert info["rc"] == 0 and info["rel_residual"] <= tol
    want = d["solution"]
    assert x.shape == want.shape
    err = np.linalg.norm(x - want) / np.linalg.norm(want)
    assert err <= bound, err
