"""Elasticity post-processing on the GPU (csrc/post.cu) against its restatement oracle/post.py,
which tests/test_cells_oracle.py pins to the reference grid's own functions: per element U,
grad U, stress, von Mises and the driver's printed fields, after a real solve."""
import numpy as np
import pytest

from multiscalefemsolver3d_b200 import fem, meshgen, meshio
from oracle import post

pytestmark = pytest.mark.gpu


def test_postprocess_matches_oracle(lib, cuda, tmp_path):
    p = meshgen.cube_elastic(n=6, jitter=0.1, n_spheres=3, contrast=20.0, rmin=0.1, rmax=0.2)
    m = p.mesh
    dofs = (3 * p.bc_nodes[:, None] + np.arange(3)).ravel().astype(np.int32)
    with fem.System(fem.ELASTIC, m.xyz, m.tets, m.mat) as S:
        S.add_traction(p.faces, p.traction)
        S.assemble_elastic(p.E, p.nu)
        S.apply_dirichlet(dofs, np.zeros(dofs.size), fem.ROW_AND_COLUMN)
        rel, it, rc = S.solve(fem.MINRES, fem.FP64, tol=1e-10, maxiter=20000)
        assert rc == 0
        u = S.get_x()
        got = S.postprocess_elastic(p.E, p.nu)
    want = post.element_fields(m.xyz, m.tets, m.mat, p.E, p.nu, u)
    np.testing.assert_allclose(got, want, rtol=1e-11, atol=1e-12 * np.abs(want).max())
    vals, names = meshio.elastic_result_fields(got)
    meshio.write_tecplot(tmp_path / "U.dat", m.xyz, m.tets, m.mat, vals, names)
    text = (tmp_path / "U.dat").read_text()
    assert f"N={m.n_nodes},  E={m.n_tets}, F=FEBLOCK ET=Tetrahedron" in text
    assert text.count("CELLCENTERED") == 6
