"""The MsFEM Order1 elasticity driver on the GPU (multiscalefemsolver3d_b200/msfem.py) against its
CPU restatement (oracle/msfem.py) on the same cell bases: macro element matrices, loads, macro
solution and the fine solution on every cell, within 1e-8 (relative to their largest entries).
The restatement's quadratures and material law are pinned against the reference's own objects
in tests/test_cells_oracle.py."""
import numpy as np
import pytest

from multiscalefemsolver3d_b200 import meshgen
from multiscalefemsolver3d_b200.cells import FP32_IR, Cells
from multiscalefemsolver3d_b200.msfem import cube_macro_boundary, msfem_elastic_driver
from oracle import msfem as om

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("spheres", [0, 6])
def test_msfem_driver_matches_oracle(lib, cuda, spheres):
    p = meshgen.cube_elastic(n=8, jitter=0.0, n_spheres=spheres, contrast=50.0, rmin=0.08, rmax=0.16, sphere_seed=5)
    cc = meshgen.cube_cells(p.mesh, p.E, p.nu, 4)
    fv, fval, items, tr = cube_macro_boundary(cc)
    cells = Cells(cc.cells)
    res = msfem_elastic_driver(cc, fv, fval, items, tr, precision=FP32_IR, tol=1e-12, cell_tol=1e-12, cells=cells)
    U, u, K, F = om.driver(cc, cells.bases(), fv, fval, items, tr, p.E[0], p.nu[0])
    np.testing.assert_allclose(res.K, K, rtol=0, atol=1e-12 * np.abs(K).max())
    np.testing.assert_allclose(res.F, F, rtol=0, atol=1e-13 * np.abs(F).max())
    assert np.abs(res.U - U).max() <= 1e-8 * np.abs(U).max()
    assert np.abs(res.u_cells - u).max() <= 1e-8 * np.abs(u).max()
    np.testing.assert_allclose(res.F.sum(axis=0), [0, 0, -1], atol=1e-12)
    assert np.all(res.U[fv] == 0)
