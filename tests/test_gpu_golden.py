"""The GPU path on the full 20^3 elasticity workload (27,783 DOF, 48,000 tets)
against the reference's own results stored in tests/golden/c1_elastic.npz."""
import os

import numpy as np
import pytest

from multiscalefemsolver3d_b200 import fem, meshgen

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("method,precision", [(fem.PCG_JACOBI, fem.FP64), (fem.MINRES, fem.FP32_IR),
                                              (fem.MINRES, fem.FP64), (fem.CG, fem.FP64)])
def test_c1_driver_matches_reference(cuda, method, precision):
    d = np.load(os.path.join(G, "c1_elastic.npz"))
    p = meshgen.cube_elastic(n=int(d["n"]), jitter=float(d["jitter"]), seed=int(d["seed"]))
    x, stats, rc = fem.fem_elastic_driver(p, method=method, precision=precision, min_residual=1e-10)
    assert rc == 0
    xr = d["x_cg"]
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-8      # the reference's CG, 1e-12
    xd = d["x_driver"]
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-8      # FEM_forElasticDeformation's own output


def test_c1_assembled_system_checksums(cuda):
    d = np.load(os.path.join(G, "c1_elastic.npz"))
    p = meshgen.cube_elastic(n=int(d["n"]), jitter=float(d["jitter"]), seed=int(d["seed"]))
    with fem.System(fem.ELASTIC, p.mesh.xyz, p.mesh.tets, p.mesh.mat) as S:
        S.add_traction(p.faces, p.traction)
        S.assemble_elastic(p.E, p.nu)
        dofs = (3 * p.bc_nodes[:, None] + np.arange(3)).ravel().astype(np.int32)
        S.apply_dirichlet(dofs, p.bc_values.ravel(), fem.ROW_AND_COLUMN)
        A = S.export_csr()
    assert A.row_ptr[-1] == int(d["nnz"])
    assert int(A.col.astype(np.int64).sum()) == int(d["col_sum"])
    assert np.abs(A.val).sum() == pytest.approx(float(d["val_abs_sum"]), rel=1e-12)
    assert np.linalg.norm(A.val) == pytest.approx(float(d["val_fro"]), rel=1e-12)
    np.testing.assert_allclose(A.F, d["F"], rtol=0, atol=1e-10 * np.abs(d["F"]).max())  # see test_golden.py
