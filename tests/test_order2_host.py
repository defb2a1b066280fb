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


def _case():
    vxyz, cv, cm = o2.graded_cells(2, 3, 0.4)
    bases = []
    for c in range(cm.n_cells):
        xyz, tets, mat, box = cm.cell(c)
        bases.append(o2.order2_bases(xyz, tets, mat, box, cm.E, cm.nu, cv[c]))
    bot = np.nonzero(np.abs(vxyz[:, 2]) < 1e-12)[0]
    top = np.nonzero(np.abs(vxyz[:, 2] - 1) < 1e-12)[0]
    side = np.nonzero(np.abs(vxyz[:, 0] - 1) < 1e-12)[0]
    groups = [(bot, (0.0, 0.0, 0.0), (1, 1, 1)), (top, (0.01, -0.02, 0.05), (1, 1, 1)),
              (side, (0.03, 0.0, 0.0), (1, 0, 0))]
    return vxyz, cv, cm, bases, groups


def test_order2_topology_macro_system_and_dirichlet_values_match_restatement(lib):
    """The product's host side of the Order2 driver (macro topology, the macro CSR summed by the
    library, the projected Dirichlet values) on the restatement's bases: the same topology, the
    same system as the restatement's dense assembly, the same fixed values, and with them the same
    macro solution.  (The GPU builds of the bases and element matrices, the Dirichlet rows and the
    solve are covered by their own GPU tests.)"""
    from multiscalefemsolver3d_b200 import order2 as p2
    vxyz, cv, cm, bases, groups = _case()
    topo = p2.macro_topology(cv, n_vertices=vxyz.shape[0])
    edges, faces, cell_faces, dofs = o2.macro_topology(cv)
    np.testing.assert_array_equal(topo.edges, edges)
    np.testing.assert_array_equal(topo.faces, faces)
    np.testing.assert_array_equal(topo.cell_faces, cell_faces)
    np.testing.assert_array_equal(topo.cell_dofs, dofs)
    K = np.stack([o2.macro_element_matrix(*cm.cell(c)[:2], bases[c], cm.cell(c)[3], cm.E[0], cm.nu[0])
                  for c in range(cm.n_cells)])
    A = p2.macro_csr(topo, K)
    dense = np.zeros((3 * topo.n_dofs,) * 2)
    for c in range(cm.n_cells):
        idx = (3 * dofs[c][:, None] + np.arange(3)).ravel()
        dense[np.ix_(idx, idx)] += K[c].transpose(0, 2, 1, 3).reshape(81, 81)
    np.testing.assert_allclose(A.to_scipy().toarray(), dense, rtol=0, atol=1e-14 * np.abs(dense).max())
    assert np.all(np.diff(A.row_ptr) % 3 == 0)            # whole 3x3 blocks per row
    got = p2.dirichlet_values(vxyz, cm, topo, bases, groups)
    want = o2.dirichlet_fixed(vxyz, cv, cm, groups, bases)
    assert [i for i, _ in got] == [i for i, _ in want]
    np.testing.assert_allclose([v for _, v in got], [v for _, v in want], rtol=0, atol=1e-13)
    # the composition: eliminate and solve the product's system, compare with the restated driver
    M = A.to_scipy().toarray()
    F = np.zeros(M.shape[0])
    for i, v in got:
        F -= M[:, i] * v
        M[:, i] = 0.0
        M[i, :] = 0.0
        M[i, i] = 1.0
        F[i] = v
    x = np.linalg.solve(M, F).reshape(-1, 3)
    xo = o2.order2_driver(vxyz, cv, cm, groups, bases=bases)
    assert np.linalg.norm(x - xo) <= 1e-11 * np.linalg.norm(xo)


def test_order2_driver_orchestration_with_stand_ins(monkeypatch, lib):
    """order2.order2_elastic_driver end to end with its two GPU objects replaced by stand-ins that
    return the restatement's bases and element matrices and solve the eliminated system exactly:
    the glue (DOF lists, the CSR from the library, the projected values, their elimination order,
    the reshape) reproduces the restated driver."""
    from multiscalefemsolver3d_b200 import cells as gcells
    from multiscalefemsolver3d_b200 import fem
    from multiscalefemsolver3d_b200 import order2 as p2
    vxyz, cv, cm, bases, groups = _case()
    K = np.stack([o2.macro_element_matrix(*cm.cell(c)[:2], bases[c], cm.cell(c)[3], cm.E[0], cm.nu[0])
                  for c in range(cm.n_cells)])

    class FakeCells:
        def __init__(self, meshes):
            assert meshes is cm

        def build_order2(self, cell_vertex, precision, tol):
            np.testing.assert_array_equal(cell_vertex, cv)
            return 0

        def order2_macro_matrices(self):
            return K

        def order2_bases(self):
            return np.concatenate(bases)

        def close(self):
            pass

    class FakeSystem:
        @classmethod
        def from_csr(cls, A, F=None, X=None):
            self = cls()
            self.A = A.to_scipy().toarray()
            self.F = np.zeros(A.n)
            return self

        def apply_dirichlet(self, dofs, vals, mode):
            assert mode == fem.ROW_AND_COLUMN
            for i, v in zip(dofs, vals):
                col = self.A[:, i].copy()
                col[i] = 0.0
                self.F -= col * v
                self.A[:, i] = 0.0
                self.A[i, :] = 0.0
                self.A[i, i] = 1.0
                self.F[i] = v

        def copy_f_to_x(self):
            pass

        def solve(self, method, precision, tol, maxiter):
            self.x = np.linalg.solve(self.A, self.F)
            return 0.0, 1, 0

        def get_x(self):
            return self.x

        def close(self):
            pass

    monkeypatch.setattr(gcells, "Cells", FakeCells)
    monkeypatch.setattr(fem.System, "from_csr", FakeSystem.from_csr)
    # groups without shared DOFs: the product eliminates each DOF once with its last value
    g2 = groups[:2]
    x, info = p2.order2_elastic_driver(cm, vxyz, cv, g2)
    xo = o2.order2_driver(vxyz, cv, cm, g2, bases=bases)
    assert info["n_dofs"] == xo.shape[0]
    assert np.linalg.norm(x - xo) <= 1e-11 * np.linalg.norm(xo)
