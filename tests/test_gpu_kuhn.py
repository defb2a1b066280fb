"""Matrix-free elasticity products on a structured Kuhn grid (csrc/kuhn.cu, csrc/kuhn.cuh).

The product formed from the tetrahedra's material codes must be the assembled matrix's: against
the oracle's assembly of the reference's element blocks (FEM_Grid.h:2125-2192, with the Dirichlet
rows and columns of FEM/FEM.h:1697-1812) at the SpMV parity bar, and against the GPU's own
assembled SELL product in both orientations, on cubes and on anisotropic boxes with several
materials (one of zero stiffness), with row-and-column and row-only Dirichlet lists.  The grid
check rejects meshes that are not the grid; the operator refuses values that are not one assembly;
the two-level solve refuses operators whose system changed after set-up."""
import numpy as np
import pytest

from multiscalefemsolver3d_b200 import fem, meshgen
from multiscalefemsolver3d_b200._lib import MsfemError

pytestmark = pytest.mark.gpu


class _Problem:
    pass


def box_problem(nx, ny, nz, size=(1.0, 1.0, 1.0), n_mat=3, seed=0):
    """A Kuhn box with random materials (material n_mat-1 has E = 0), u = 0 on z = 0, traction on
    the top faces."""
    m = meshgen.kuhn_box(nx, ny, nz, size=size)
    rng = np.random.default_rng(seed)
    m.mat = rng.integers(0, n_mat, m.n_tets).astype(np.int32)
    p = _Problem()
    p.mesh = m
    p.E = np.concatenate([rng.uniform(1.0, 100.0, n_mat - 1), [0.0]])
    p.nu = rng.uniform(0.2, 0.4, n_mat)
    p.bc_nodes = meshgen.nodes_on_plane(m, 2, 0.0)
    p.bc_mask = np.full(p.bc_nodes.size, 7, dtype=np.int32)
    p.bc_values = np.zeros((p.bc_nodes.size, 3))
    p.faces, p.face_elem = meshgen.boundary_faces_on_plane(m, 2, size[2])
    p.traction = np.tile([0.0, 0.0, -1.0], (p.faces.shape[0], 1))
    return p


def _dofs(p):
    return (3 * p.bc_nodes[:, None] + np.arange(3)).ravel().astype(np.int32)


def _system(p, textbook=False, mode=fem.ROW_AND_COLUMN, dofs=None):
    S = fem.System(fem.ELASTIC, p.mesh.xyz, p.mesh.tets, p.mesh.mat)
    S.add_traction(p.faces, p.traction)
    if textbook:
        S.assemble_elastic_textbook(p.E, p.nu)
    else:
        S.assemble_elastic(p.E, p.nu)
    d = _dofs(p) if dofs is None else dofs
    S.apply_dirichlet(d, np.zeros(d.size), mode)
    return S


CASES = {
    "cube-spheres": lambda: meshgen.cube_elastic(n=8, jitter=0.0, n_spheres=4, contrast=50.0, rmin=0.1, rmax=0.2),
    "box-3-materials": lambda: box_problem(5, 4, 3, size=(1.0, 2.0, 0.5)),
    "box-tall": lambda: box_problem(2, 3, 11, size=(0.3, 0.4, 2.0), n_mat=2, seed=1),
}


@pytest.mark.parametrize("case", list(CASES))
def test_product_matches_the_oracle(cuda, port, case):
    """The reference's orientation, Dirichlet rows and columns: the oracle's assembled matrix
    times x, at the SpMV parity bar."""
    p = CASES[case]()
    n = p.mesh.meta.get("box", (p.mesh.n,) * 3)
    with _system(p) as S:
        S.set_kuhn_grid(*n)
        A = port.elastic_system(p, stage=1)
        x = np.random.default_rng(3).normal(size=S.n_rows)
        y = S.kuhn_spmv(x)
        yo = port.spmv(A, x)
        np.testing.assert_allclose(y, yo, rtol=0, atol=1e-13 * np.abs(A.val).max() * np.abs(x).max() * 45)
        ya = S.spmv(x)
        assert np.linalg.norm(y - ya) <= 1e-13 * np.linalg.norm(ya)


@pytest.mark.parametrize("textbook", [False, True], ids=["reference", "textbook"])
@pytest.mark.parametrize("mode", [fem.ROW_AND_COLUMN, fem.ROW_ONLY], ids=["rows-and-columns", "rows-only"])
def test_product_matches_the_assembled_matrix(cuda, textbook, mode):
    p = box_problem(6, 5, 4, size=(1.5, 1.0, 0.8), n_mat=4, seed=2)
    rng = np.random.default_rng(5)
    dofs = rng.permutation(_dofs(p))[: 3 * p.bc_nodes.size // 2].astype(np.int32)  # unsorted, partial
    if mode == fem.ROW_AND_COLUMN:
        dofs = np.sort(dofs)  # the column walk of an unsorted list leaves columns in (reference quirk)
    with _system(p, textbook, mode, dofs) as S:
        S.set_kuhn_grid(6, 5, 4)
        for seed in range(3):
            x = np.random.default_rng(seed).normal(size=S.n_rows)
            y, ya = S.kuhn_spmv(x), S.spmv(x)
            assert np.linalg.norm(y - ya) <= 1e-13 * np.linalg.norm(ya)
            assert np.abs(y - ya).max() <= 1e-12 * np.abs(ya).max()


def test_unsorted_column_list_is_refused(cuda):
    """With an unsorted Dirichlet list the reference's one-pointer column walk leaves some columns
    in the matrix; the matrix-free product would eliminate them, so its check refuses it."""
    p = box_problem(4, 4, 4, seed=3)
    dofs = _dofs(p)[::-1].copy()
    with _system(p, False, fem.ROW_AND_COLUMN, dofs) as S:
        S.set_kuhn_grid(4)
        A = S.export_csr()
        rows = np.repeat(np.arange(A.n), np.diff(A.row_ptr))
        left = np.isin(A.col, dofs) & (rows != A.col) & (A.val != 0.0)
        if not left.any():
            pytest.skip("the walk eliminated every column of this list")
        with pytest.raises(MsfemError, match="differs from the assembled"):
            S.kuhn_spmv(np.ones(S.n_rows))


def test_grid_check_rejects_other_meshes(cuda):
    p = meshgen.cube_elastic(n=4, jitter=0.0)
    m = p.mesh
    with fem.System(fem.ELASTIC, m.xyz, m.tets, m.mat) as S:
        with pytest.raises(MsfemError, match="do not give"):
            S.set_kuhn_grid(4, 4, 5)
        S.set_kuhn_grid(4)
    j = meshgen.cube_elastic(n=4, jitter=0.2).mesh
    with fem.System(fem.ELASTIC, j.xyz, j.tets, j.mat) as S:
        with pytest.raises(MsfemError, match="not at its grid position"):
            S.set_kuhn_grid(4)
    t = m.tets.copy()
    t[7, [1, 2]] = t[7, [2, 1]]
    with fem.System(fem.ELASTIC, m.xyz, t, m.mat) as S:
        with pytest.raises(MsfemError, match="tetrahedron 7 "):
            S.set_kuhn_grid(4)
    mat = m.mat.copy()
    mat[11] = 64
    with fem.System(fem.ELASTIC, m.xyz, m.tets, mat) as S:
        with pytest.raises(MsfemError, match="tetrahedron 11 "):
            S.set_kuhn_grid(4)


def test_values_must_be_one_assembly(cuda):
    p = box_problem(3, 3, 3, seed=4)
    with fem.System(fem.ELASTIC, p.mesh.xyz, p.mesh.tets, p.mesh.mat) as S:
        S.set_kuhn_grid(3)
        x = np.random.default_rng(0).normal(size=S.n_rows)
        with pytest.raises(MsfemError, match="not one"):
            S.kuhn_spmv(x)                      # nothing assembled
        S.assemble_elastic(p.E, p.nu)
        y1 = S.kuhn_spmv(x)
        S.assemble_elastic(p.E, p.nu)           # twice: the values are 2A
        with pytest.raises(MsfemError, match="not one"):
            S.kuhn_spmv(x)
        S.clear()
        S.assemble_elastic(p.E, p.nu)
        np.testing.assert_array_equal(S.kuhn_spmv(x), y1)   # deterministic


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("textbook", [False, True], ids=["reference", "textbook"])
def test_scaled_fp32_product_on_pre_scaled_input(cuda, case, textbook):
    """The smoother's kernel (input s x with the eliminated columns zero, staged as it is) on cubes
    and anisotropic boxes, both orientations: S A S x equals the assembled FP32 product at the FP32
    bar, and its set-up check compared it bit for bit with the staged-scale kernel (it would have
    raised otherwise); repeated calls agree bit for bit."""
    p = CASES[case]()
    n = p.mesh.meta.get("box", (p.mesh.n,) * 3)
    with _system(p, textbook=textbook) as S:
        S.set_kuhn_grid(*n)
        x = np.random.default_rng(3).standard_normal(S.n_rows).astype(np.float32)
        y = S.kuhn_spmv_scaled32(x)
        ya = S.spmv_scaled32(x)
        assert np.linalg.norm(y - ya) <= 1e-5 * np.linalg.norm(ya)
        np.testing.assert_array_equal(S.kuhn_spmv_scaled32(x), y)


def test_two_level_refuses_a_changed_system(cuda):
    from multiscalefemsolver3d_b200.cells import FP64, Cells
    from multiscalefemsolver3d_b200.twolevel import TwoLevel
    p = meshgen.cube_elastic(n=8, jitter=0.0, n_spheres=3, contrast=10.0, rmin=0.1, rmax=0.2)
    dofs = _dofs(p)
    S = _system(p)
    K = _system(p, textbook=True)
    S.set_kuhn_grid(8)
    K.set_kuhn_grid(8)
    cc = meshgen.cube_cells(p.mesh, p.E, p.nu, 4)
    cells = Cells(cc.cells)
    assert cells.build_bases(FP64, 1e-12) == 0
    T = TwoLevel(S, cells, cc, dofs)
    T.set_smoother(K, degree=3, matrix_free=True)
    T.set_matrix_free(True)
    S.set_x(np.zeros(S.n_rows))
    rel, it, _, rc = T.solve(tol=1e-8, maxiter=20000, precision=FP64)
    assert rc == 0 and rel <= 1e-8
    K.apply_dirichlet(dofs, np.zeros(dofs.size), fem.ROW_AND_COLUMN)   # values changed (same values)
    with pytest.raises(MsfemError, match="changed after it was set up"):
        T.solve(tol=1e-8, maxiter=20000, precision=FP64)
    T.close()
