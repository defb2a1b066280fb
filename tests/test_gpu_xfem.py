"""Cracked conduction assembled on the GPU (csrc/xfem.cu) against its restatement oracle/xfem.py:
the same matrix (pattern exact, values within 1e-12 of the largest), the solution of the Dirichlet
problem within 1e-8 of the exact one (GMRES(50) with FP32 Krylov vectors in FP64 refinement),
and a crack through the whole cube decoupling the halves exactly."""
import numpy as np
import pytest

from multiscalefemsolver3d_b200 import fem, meshgen, xfem
from oracle import xfem as ox

pytestmark = pytest.mark.gpu


def test_xfem_matrix_and_solution_match_oracle(lib, cuda):
    mesh, cr, nodes, vals = xfem.cube_cracked(n=10, n_cracks=8, seed=3, rmin=0.1, rmax=0.3)
    S, enr = xfem.build_system(mesh, cr)
    assert enr.n_enriched > 0
    A = S.export_csr()
    B = ox.assemble(mesh.xyz, mesh.tets, np.ones(mesh.n_tets), cr, enr)
    B.sort_indices()
    np.testing.assert_array_equal(A.row_ptr, B.indptr)
    np.testing.assert_array_equal(A.col, B.indices)
    np.testing.assert_allclose(A.val, B.data, rtol=0, atol=1e-12 * np.abs(B.data).max())
    S.apply_dirichlet(nodes, vals, fem.ROW_AND_COLUMN)
    S.copy_f_to_x()
    rel, it, rc = S.solve(fem.GMRES, fem.FP32_IR, tol=1e-10, maxiter=20000, restart=50)
    assert rc == 0
    x = ox.solve_dirichlet(B, nodes, vals)
    assert np.linalg.norm(S.get_x() - x) <= 1e-8 * np.linalg.norm(x)
    S.close()


def test_xfem_full_crack_decouples_on_gpu(lib, cuda):
    mesh = meshgen.kuhn_cube(8, jitter=0.05, seed=1)
    cr = xfem.Cracks(centre=np.array([[0.5, 0.5, 0.53]]), normal=np.array([[0.0, 0.0, 1.0]]), radius=np.array([10.0]))
    S, enr = xfem.build_system(mesh, cr)
    lo = meshgen.nodes_on_plane(mesh, 2, 0.0)
    hi = meshgen.nodes_on_plane(mesh, 2, 1.0)
    S.apply_dirichlet(np.concatenate([lo, hi]).astype(np.int32), np.concatenate([np.ones(lo.size), np.zeros(hi.size)]),
                      fem.ROW_AND_COLUMN)
    S.copy_f_to_x()
    rel, it, rc = S.solve(fem.GMRES, fem.FP64, tol=1e-12, maxiter=20000, restart=50)
    assert rc == 0
    T = S.get_x()[:mesh.n_nodes]
    below = mesh.xyz[:, 2] < 0.53
    np.testing.assert_allclose(T[below], 1.0, atol=1e-9)
    np.testing.assert_allclose(T[~below], 0.0, atol=1e-9)
    S.close()
