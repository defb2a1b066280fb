"""GPU path vs the oracle on the same seeded inputs, through the C ABI.

Bars: sparsity pattern, DOF numbering and Dirichlet structure bit-exact;
assembled values within 1e-12 of the largest entry (different but equally
exact element formulas, different summation order); solutions within 1e-8
relative L2 of the oracle's FP64 solution (the reference's stated tolerance).
"""
import numpy as np
import pytest

from multiscalefemsolver3d_b200 import fem, meshgen

pytestmark = pytest.mark.gpu

VAL_TOL = 1e-12   # assembled values: atol relative to max |a_ij|
SOL_TOL = 1e-8    # solutions: relative L2


def elastic_system(p):
    S = fem.System(fem.ELASTIC, p.mesh.xyz, p.mesh.tets, p.mesh.mat)
    S.add_traction(p.faces, p.traction)
    S.assemble_elastic(p.E, p.nu)
    return S


def elastic_dofs(p):
    dofs, vals = [], []
    for i, node in enumerate(p.bc_nodes):
        for c in range(3):
            if p.bc_mask[i] & (1 << c):
                dofs.append(3 * node + c)
                vals.append(p.bc_values[i, c])
    return np.array(dofs, dtype=np.int32), np.array(vals)


def scalar_system(p):
    S = fem.System(fem.SCALAR, p.mesh.xyz, p.mesh.tets, p.mesh.mat)
    S.assemble_scalar(p.sigma)
    return S


def assert_system_equal(G, O):
    np.testing.assert_array_equal(G.row_ptr, O.row_ptr)
    np.testing.assert_array_equal(G.col, O.col)
    scale = np.abs(O.val).max()
    np.testing.assert_allclose(G.val, O.val, rtol=0, atol=VAL_TOL * scale)
    np.testing.assert_allclose(G.F, O.F, rtol=0, atol=VAL_TOL * max(1.0, np.abs(O.F).max()))
    np.testing.assert_allclose(G.X, O.X, rtol=0, atol=VAL_TOL * max(1.0, np.abs(O.X).max()))


def assert_dirichlet_structure(G, dofs, columns=True):
    """Dirichlet rows are exact unit rows; eliminated columns are exact zeros off the diagonal."""
    bc = np.unique(dofs)
    for d in bc:
        a, b = G.row_ptr[d], G.row_ptr[d + 1]
        np.testing.assert_array_equal(G.val[a:b], (G.col[a:b] == d).astype(float))
    if columns:
        hit = np.isin(G.col, bc)
        rows = np.repeat(np.arange(G.n), np.diff(G.row_ptr))
        assert np.all(G.val[hit & (rows != G.col)] == 0.0)


@pytest.mark.parametrize("n,spheres", [(3, 0), (6, 3), (10, 8)])
def test_elastic_assembly_and_dirichlet(cuda, port, n, spheres):
    p = meshgen.cube_elastic(n=n, n_spheres=spheres, contrast=50.0, rmin=0.08, rmax=0.15, sphere_seed=11)
    with elastic_system(p) as S:
        assert_system_equal(S.export_csr(), port.elastic_system(p, stage=0))
        d, v = elastic_dofs(p)
        S.apply_dirichlet(d, v, fem.ROW_AND_COLUMN)
        G = S.export_csr()
        assert_system_equal(G, port.elastic_system(p, stage=1))
        assert_dirichlet_structure(G, d)  # the elasticity list is sorted: every column is eliminated


@pytest.mark.parametrize("n,spheres", [(4, 0), (9, 6), (16, 12)])
def test_scalar_assembly_and_dirichlet(cuda, port, n, spheres):
    """Includes the reference's unsorted two-type boundary list (x=0 then x=1)."""
    p = meshgen.cube_scalar(n=n, n_spheres=spheres, rmin=0.06, rmax=0.12, contrast=100.0)
    with scalar_system(p) as S:
        assert_system_equal(S.export_csr(), port.scalar_system(p, stage=0))
        S.apply_dirichlet(p.bc_nodes, p.bc_values, fem.ROW_AND_COLUMN)
        S.copy_f_to_x()
        assert_system_equal(S.export_csr(), port.scalar_system(p, stage=1))


def test_shuffled_and_duplicate_boundary_lists(cuda, port):
    p = meshgen.cube_scalar(n=6, n_spheres=0)
    rng = np.random.default_rng(3)
    perm = rng.permutation(p.bc_nodes.size)
    nodes = np.concatenate([p.bc_nodes[perm], p.bc_nodes[perm[:5]]]).astype(np.int32)
    vals = np.concatenate([p.bc_values[perm], np.arange(5, dtype=float)])
    p.bc_nodes, p.bc_values = nodes, vals
    with scalar_system(p) as S:
        S.apply_dirichlet(p.bc_nodes, p.bc_values, fem.ROW_AND_COLUMN)
        S.copy_f_to_x()
        assert_system_equal(S.export_csr(), port.scalar_system(p, stage=1))


def test_row_only_dirichlet(cuda, port):
    """FEM/FEM.h:297-324: rows replaced, columns untouched (nonsymmetric system)."""
    p = meshgen.cube_scalar(n=5, n_spheres=0)
    with scalar_system(p) as S:
        before = S.export_csr()
        S.apply_dirichlet(p.bc_nodes, p.bc_values, fem.ROW_ONLY)
        after = S.export_csr()
    bc = set(p.bc_nodes.tolist())
    for i in range(after.n):
        a, b = after.row_ptr[i], after.row_ptr[i + 1]
        if i in bc:
            np.testing.assert_array_equal(after.val[a:b], (after.col[a:b] == i).astype(float))
        else:
            np.testing.assert_array_equal(after.val[a:b], before.val[a:b])


def test_spmv_matches_oracle(cuda, port):
    p = meshgen.cube_elastic(n=7, n_spheres=3, contrast=20.0, rmin=0.1, rmax=0.2)
    with elastic_system(p) as S:
        d, v = elastic_dofs(p)
        S.apply_dirichlet(d, v, fem.ROW_AND_COLUMN)
        A = S.export_csr()
        x = np.random.default_rng(0).normal(size=S.n_rows)
        y = S.spmv(x)
        np.testing.assert_allclose(y, port.spmv(A, x), rtol=0, atol=1e-13 * np.abs(A.val).max() * np.abs(x).max() * 45)


@pytest.mark.parametrize("kind", ["scalar", "elastic"])
def test_fp32_scaled_operator(cuda, kind):
    """The FP32 inner solves apply D^-1/2 A D^-1/2 from a FP32 copy; compare with the FP64
    matrix scaled on the host (FP32 rounding of the values and of the sums)."""
    if kind == "elastic":
        p = meshgen.cube_elastic(n=7, n_spheres=3, contrast=20.0, rmin=0.1, rmax=0.2)
        S = elastic_system(p)
        d, v = elastic_dofs(p)
        S.apply_dirichlet(d, v, fem.ROW_AND_COLUMN)
    else:
        p = meshgen.cube_scalar(n=9, n_spheres=5, rmin=0.06, rmax=0.12)
        S = scalar_system(p)
        S.apply_dirichlet(p.bc_nodes, p.bc_values, fem.ROW_AND_COLUMN)
    with S:
        A = S.export_csr().to_scipy()
        sc = 1.0 / np.sqrt(np.abs(A.diagonal()))
        x = np.random.default_rng(1).normal(size=S.n_rows).astype(np.float32)
        y = S.spmv_scaled32(x)
        yr = sc * (A @ (sc * x.astype(np.float64)))
        assert np.abs(y - yr).max() <= 1e-5 * np.abs(yr).max()


def reference_solution(port, A):
    x, res, _ = port.cg(A, tol=1e-14, maxiter=200000)
    return x


@pytest.mark.parametrize("method,precision", [
    (fem.CG, fem.FP64), (fem.PCG_JACOBI, fem.FP64), (fem.BICGSTAB, fem.FP64), (fem.GMRES, fem.FP64),
    (fem.GMRES, fem.FP32_IR), (fem.MINRES, fem.FP64), (fem.MINRES, fem.FP32_IR)])
def test_elastic_solvers(cuda, port, method, precision):
    p = meshgen.cube_elastic(n=8, n_spheres=4, contrast=10.0, rmin=0.1, rmax=0.2)
    with elastic_system(p) as S:
        d, v = elastic_dofs(p)
        S.apply_dirichlet(d, v, fem.ROW_AND_COLUMN)
        A = S.export_csr()
        rel, it, rc = S.solve(method, precision, tol=1e-10, maxiter=50000, restart=40)
        assert rc == 0, (rel, it)
        assert rel <= 1e-10 * 1.5
        x = S.get_x()
    xr = reference_solution(port, A)
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < SOL_TOL


@pytest.mark.parametrize("method,precision", [
    (fem.PCG_JACOBI, fem.FP64), (fem.CG, fem.FP64), (fem.PCG_JACOBI, fem.FP32_IR), (fem.GMRES, fem.FP64),
    (fem.GMRES, fem.FP32_IR), (fem.MINRES, fem.FP64), (fem.MINRES, fem.FP32_IR)])
def test_scalar_solvers(cuda, port, method, precision):
    p = meshgen.cube_scalar(n=14, n_spheres=10, rmin=0.05, rmax=0.1, contrast=100.0)
    with scalar_system(p) as S:
        S.apply_dirichlet(p.bc_nodes, p.bc_values, fem.ROW_AND_COLUMN)
        S.copy_f_to_x()
        A = S.export_csr()
        rel, it, rc = S.solve(method, precision, tol=1e-10, maxiter=50000, restart=40)
        assert rc == 0
        x = S.get_x()
    xr = reference_solution(port, A)
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < SOL_TOL


def test_fp32_refinement_needs_the_jacobi_inner_solver(cuda):
    p = meshgen.cube_scalar(n=4, n_spheres=0)
    with scalar_system(p) as S:
        S.apply_dirichlet(p.bc_nodes, p.bc_values, fem.ROW_AND_COLUMN)
        with pytest.raises(fem._lib.MsfemError) as e:
            S.solve(fem.CG, fem.FP32_IR, tol=1e-8)
        assert e.value.rc == -1


def test_pcg_follows_the_oracle_iteration(cuda, port):
    """Jacobi-PCG on the GPU is the reference's PCG loop (MSG_PreconditioningSSOR with
    M = diag(A)): the same iteration count up to the rounding of the dot products (tree vs
    serial sums) and the same iterate."""
    p = meshgen.cube_elastic(n=10)
    with elastic_system(p) as S:
        d, v = elastic_dofs(p)
        S.apply_dirichlet(d, v, fem.ROW_AND_COLUMN)
        A = S.export_csr()
        rel, it, rc = S.solve(fem.PCG_JACOBI, fem.FP64, tol=1e-10, maxiter=100000)
        x = S.get_x()
    xo, reso, ito = port.pcg_jacobi(A, tol=1e-10)
    assert abs(it - ito) <= max(2, int(0.02 * ito))
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-9


def test_solves_are_deterministic(cuda):
    p = meshgen.cube_scalar(n=12, n_spheres=6, rmin=0.05, rmax=0.1)
    xs = []
    for _ in range(2):
        with scalar_system(p) as S:
            S.apply_dirichlet(p.bc_nodes, p.bc_values, fem.ROW_AND_COLUMN)
            S.copy_f_to_x()
            S.solve(fem.PCG_JACOBI, fem.FP64, tol=1e-10)
            xs.append(S.get_x())
    np.testing.assert_array_equal(xs[0], xs[1])


def test_zero_stiffness_material_contributes_nothing(cuda, port):
    p = meshgen.cube_elastic(n=5, n_spheres=2, contrast=1.0, rmin=0.15, rmax=0.25)
    p.E = np.array([1.0, 0.0])  # material 1 has E = 0 -> skipped (FEM/FEM.h:1355-1363)
    with elastic_system(p) as S:
        assert_system_equal(S.export_csr(), port.elastic_system(p, stage=0))


def test_bad_inputs_return_errors(cuda):
    m = meshgen.kuhn_cube(3)
    bad = m.tets.copy()
    bad[5, 2] = m.n_nodes + 7
    with pytest.raises(fem._lib.MsfemError) as e:
        fem.System(fem.SCALAR, m.xyz, bad)
    assert e.value.rc == -1
    with fem.System(fem.SCALAR, m.xyz, m.tets) as S:
        with pytest.raises(fem._lib.MsfemError):
            S.assemble_scalar(np.array([]))
        mat = np.zeros(m.n_tets, dtype=np.int32)
    with fem.System(fem.SCALAR, m.xyz, m.tets, mat + 3) as S:
        with pytest.raises(fem._lib.MsfemError):
            S.assemble_scalar([1.0])
    with fem.System(fem.SCALAR, m.xyz, m.tets) as S:
        S.assemble_scalar([1.0])
        with pytest.raises(fem._lib.MsfemError):
            S.apply_dirichlet(np.array([0, m.n_nodes], dtype=np.int32), np.zeros(2))
        # the handle stays usable after a rejected call
        S.apply_dirichlet(np.array([0], dtype=np.int32), np.zeros(1))
        S.add_rhs(np.ones(m.n_nodes))
        rel, it, rc = S.solve(fem.PCG_JACOBI, fem.FP64, tol=1e-10)
        assert rc == 0
