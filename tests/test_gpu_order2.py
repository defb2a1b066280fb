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
    matrices, the macro system, the projected Dirichlet values, Dirichlet rows and
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


def _graded_case():
    vxyz, cv, cm = o2.graded_cells(2, 3, 0.4)
    bot = np.nonzero(np.abs(vxyz[:, 2]) < 1e-12)[0]
    top = np.nonzero(np.abs(vxyz[:, 2] - 1) < 1e-12)[0]
    side = np.nonzero(np.abs(vxyz[:, 0] - 1) < 1e-12)[0]
    groups = [(bot, (0.0, 0.0, 0.0), (1, 1, 1)), (top, (0.01, -0.02, 0.05), (1, 1, 1)),
              (side, (0.03, 0.0, 0.0), (1, 0, 0))]
    return vxyz, cv, cm, groups


def test_order2_macro_system_on_device_is_the_cell_sum(lib, cuda):
    """msfem_cells_order2_macro_system: the scalar rows 3 d + c hold whole 3 x 3 blocks of the DOF
    portrait (o2.macro_portrait, the rule pinned against the reference's own portrait in
    tests/test_order2_oracle.py), diagonal in place, and every value is the sum of the cells'
    element matrices (msfem_cells_order2_macro_matrices of the same build) in cell order: bit for
    bit the dense sum."""
    from multiscalefemsolver3d_b200 import order2 as p2
    vxyz, cv, cm, _ = _graded_case()
    topo = p2.macro_topology(cv, n_vertices=vxyz.shape[0])
    c = gcells.Cells(cm)
    try:
        assert c.build_order2(cv, FP64, 1e-10) == 0
        K = c.order2_macro_matrices()
        S = p2.macro_system(c, topo)
        A = S.export_csr()
        S.close()
    finally:
        c.close()
    n = 3 * topo.n_dofs
    assert A.n == n
    dense = np.zeros((n, n))
    for k in range(cm.n_cells):
        idx = (3 * topo.cell_dofs[k][:, None] + np.arange(3)).ravel()
        dense[np.ix_(idx, idx)] += K[k].transpose(0, 2, 1, 3).reshape(81, 81)
    rule = o2.macro_portrait(topo.cell_dofs, topo.n_dofs)
    for r in range(n):
        cols = A.col[A.row_ptr[r]:A.row_ptr[r + 1]]
        np.testing.assert_array_equal(cols, (3 * rule[r // 3][:, None] + np.arange(3)).ravel())
        np.testing.assert_array_equal(A.val[A.row_ptr[r]:A.row_ptr[r + 1]], dense[r, cols])


def test_order2_dirichlet_projection_on_device_matches_oracle(lib, cuda):
    """msfem_cells_order2_dirichlet: the L2-projected values of three groups (two faces of the
    cube, one with a single taken component, sharing edges) on the device against the
    restatement's projection (oracle/order2.py dirichlet_fixed, pinned against the reference's
    whole Order2 driver) on the same GPU bases; the face bubbles hold 0."""
    from multiscalefemsolver3d_b200 import order2 as p2
    vxyz, cv, cm, groups = _graded_case()
    topo = p2.macro_topology(cv, n_vertices=vxyz.shape[0])
    lay = p2.dirichlet_layout(topo, groups)
    c = gcells.Cells(cm)
    try:
        assert c.build_order2(cv, FP64, 1e-11) == 0
        allb = c.order2_bases()
        P = p2.dirichlet_projection(c, topo, vxyz, lay)
    finally:
        c.close()
    bases = [allb[cm.node_off[k]:cm.node_off[k + 1]] for k in range(cm.n_cells)]
    want = o2.dirichlet_fixed(vxyz, cv, cm, groups, bases)
    j = 0
    scale = max(abs(v) for _, v in want)
    for g, (_, _, take) in enumerate(groups):
        for k in range(lay.group_dof_off[g], lay.group_dof_off[g + 1]):
            for comp in range(3):
                if take[comp]:
                    d, v = want[j]
                    assert d == 3 * int(lay.group_dofs[k]) + comp
                    assert abs(P[k, comp] - v) <= 1e-12 * scale, (g, k, comp, P[k, comp], v)
                    j += 1
    assert j == len(want)
    nv, ne = topo.n_vertices, len(topo.edges)
    bubbles = lay.group_dofs >= nv + ne
    assert bubbles.any() and np.all(P[bubbles] == 0.0)
