"""A matrix imported in the reference's CSSD_Matrix layout (msfem_system_from_cssd) runs through
the same GPU solvers as an assembled one: importing the export of an assembled system gives the
same matrix (export bit-identical) and the same iterates; unsorted lists are sorted, bad
columns are rejected; the imported system has no mesh to assemble from."""
import numpy as np
import pytest
import scipy.sparse.linalg as spl

from multiscalefemsolver3d_b200 import fem, meshgen
from multiscalefemsolver3d_b200._lib import MsfemError

pytestmark = pytest.mark.gpu


def _scalar_system():
    p = meshgen.cube_scalar(n=10, n_spheres=6, contrast=50.0, rmin=0.05, rmax=0.15, sphere_seed=3)
    S = fem.System(fem.SCALAR, p.mesh.xyz, p.mesh.tets, p.mesh.mat)
    S.assemble_scalar(p.sigma)
    S.apply_dirichlet(p.bc_nodes, p.bc_values, fem.ROW_AND_COLUMN)
    S.copy_f_to_x()
    return S


@pytest.mark.parametrize("method", [fem.CG, fem.PCG_JACOBI, fem.GMRES])
def test_imported_cssd_matches_assembled_system(lib, cuda, method):
    S = _scalar_system()
    A = S.export_csr()
    T = fem.System.from_csr(A, F=A.F, X=A.X)
    B = T.export_csr()
    np.testing.assert_array_equal(B.row_ptr, A.row_ptr)
    np.testing.assert_array_equal(B.col, A.col)
    np.testing.assert_array_equal(B.val, A.val)
    r1, it1, rc1 = S.solve(method, fem.FP64, tol=1e-10, maxiter=20000)
    r2, it2, rc2 = T.solve(method, fem.FP64, tol=1e-10, maxiter=20000)
    assert rc1 == 0 and rc2 == 0 and it1 == it2
    np.testing.assert_array_equal(S.get_x(), T.get_x())
    x = spl.spsolve(A.to_scipy().tocsc(), A.F)
    assert np.linalg.norm(T.get_x() - x) <= 1e-8 * np.linalg.norm(x)
    S.close()
    T.close()


def test_import_sorts_rows_and_rejects_bad_columns(lib, cuda):
    diag = np.array([4.0, 4.0, 4.0])
    # row 2's lower list given out of order
    T = fem.System.from_cssd(diag, [[], [0], [1, 0]], [[], [-1.0], [-1.0, -0.5]], [[1, 2], [2], []],
                             [[-1.0, -0.5], [-1.0], []], F=np.ones(3))
    B = T.export_csr()
    np.testing.assert_array_equal(B.col, [0, 1, 2, 0, 1, 2, 0, 1, 2])
    np.testing.assert_array_equal(B.val, [4.0, -1.0, -0.5, -1.0, 4.0, -1.0, -0.5, -1.0, 4.0])
    rel, it, rc = T.solve(fem.CG, fem.FP64, tol=1e-12, maxiter=100)
    assert rc == 0
    np.testing.assert_allclose(B.to_scipy() @ T.get_x(), np.ones(3), atol=1e-11)
    with pytest.raises(MsfemError, match="no mesh"):
        T.assemble_scalar(np.array([1.0]))
    T.close()
    with pytest.raises(MsfemError, match="lists column"):
        fem.System.from_cssd(diag, [[], [1], []], [[], [1.0], []], [[], [], []], [[], [], []])
    with pytest.raises(MsfemError, match="twice"):
        fem.System.from_cssd(diag, [[], [0, 0], []], [[], [1.0, 1.0], []], [[], [], []], [[], [], []])
