"""The oracle is pinned before it is trusted.

The C restatement (oracle/femoracle.c) is checked against the reference's own
code compiled in place (oracle/_ref, built from the reference sources by
oracle/Makefile): element matrices, portraits, assembled systems before and
after boundary conditions, and every reference solver iterate for iterate.
"""
import numpy as np
import pytest

from multiscalefemsolver3d_b200 import meshgen

UNIT_TET = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=float)


def test_unit_tet_known_answers(port):
    # E = 1, nu = 0.3 on the unit tetrahedron: lambda = 0.5769.., mu = 0.3846.., V = 1/6.
    # A[0][1] = V * (lambda g1 (x) g0 + mu g0 (x) g1 + mu (g0.g1) I) with g0 = (-1,-1,-1), g1 = (1,0,0)
    K = port.elastic_local(UNIT_TET, 1.0, 0.3)
    lam, mu, V = 0.3 / 0.7 * (0.7 / (1.3 * 0.4)), 0.4 / 1.4 * (0.7 / (1.3 * 0.4)), 1.0 / 6.0
    assert K[0, 1, 0, 0] == pytest.approx(-(lam + 2 * mu) * V, rel=1e-14)
    assert K[0, 1, 0, 1] == pytest.approx(-lam * V, rel=1e-14)   # -0.09615: the reference's orientation
    assert K[0, 1, 1, 0] == pytest.approx(-mu * V, rel=1e-14)    # -0.06410
    assert K[0, 1, 1, 1] == pytest.approx(-mu * V, rel=1e-14)
    # block symmetry of the whole element matrix, A[J][I] = A[I][J]^T
    for I in range(4):
        for J in range(4):
            np.testing.assert_array_equal(K[I, J], K[J, I].T)
    # rigid translations are in the kernel
    assert np.abs(K.sum(axis=1)).max() < 1e-14
    S = port.scalar_local(UNIT_TET, 2.0)
    np.testing.assert_allclose(S.sum(axis=1), 0, atol=1e-15)
    assert S[0, 0] == pytest.approx(2.0 * 3 / 6.0)


def test_local_matrices_match_reference(port, ref):
    rng = np.random.default_rng(5)
    for _ in range(20):
        t = UNIT_TET * rng.uniform(0.2, 3.0) + rng.normal(0, 0.15, (4, 3)) + rng.uniform(-2, 2, 3)
        E, nu = rng.uniform(0.5, 200.0), rng.uniform(0.05, 0.45)
        Kr, Kp = ref.elastic_local(t, E, nu), port.elastic_local(t, E, nu)
        np.testing.assert_allclose(Kp, Kr, rtol=0, atol=1e-12 * np.abs(Kr).max())
        s = rng.uniform(0.1, 100.0)
        Sr, Sp = ref.scalar_local(t, s), port.scalar_local(t, s)
        np.testing.assert_allclose(Sp, Sr, rtol=0, atol=1e-13 * np.abs(Sr).max())


def _same_pattern(a, b):
    np.testing.assert_array_equal(a.row_ptr, b.row_ptr)
    np.testing.assert_array_equal(a.col, b.col)


@pytest.mark.parametrize("stage", [0, 1])
@pytest.mark.parametrize("n,spheres", [(3, 0), (5, 4)])
def test_elastic_system_matches_reference(port, ref, stage, n, spheres):
    p = meshgen.cube_elastic(n=n, n_spheres=spheres, contrast=50.0, rmin=0.1, rmax=0.2, sphere_seed=3)
    A, _ = ref.elastic_system(p, stage=stage)
    B = port.elastic_system(p, stage=stage)
    _same_pattern(A, B)
    scale = np.abs(A.val).max()
    np.testing.assert_allclose(B.val, A.val, rtol=0, atol=1e-13 * scale)
    np.testing.assert_allclose(B.F, A.F, rtol=0, atol=1e-14 * max(1.0, np.abs(A.F).max()))
    np.testing.assert_array_equal(B.X, A.X)


@pytest.mark.parametrize("stage", [0, 1])
def test_scalar_system_matches_reference(port, ref, stage):
    p = meshgen.cube_scalar(n=7, n_spheres=5, rmin=0.08, rmax=0.15, contrast=100.0)
    A, _ = ref.scalar_system(p, stage=stage)
    B = port.scalar_system(p, stage=stage)
    _same_pattern(A, B)
    np.testing.assert_allclose(B.val, A.val, rtol=0, atol=1e-13 * np.abs(A.val).max())
    np.testing.assert_allclose(B.F, A.F, rtol=0, atol=1e-14)
    np.testing.assert_allclose(B.X, A.X, rtol=0, atol=1e-14)


def test_unsorted_boundary_list_walk(port, ref):
    """The scalar driver's boundary list (x=0 face, then x=1 face) is not sorted;
    the reference's forward-only walk then leaves most x=1 columns in place."""
    p = meshgen.cube_scalar(n=6, n_spheres=0)
    A, _ = ref.scalar_system(p, stage=1)
    B = port.scalar_system(p, stage=1)
    _same_pattern(A, B)
    np.testing.assert_allclose(B.val, A.val, rtol=0, atol=1e-13)
    M = A.to_scipy().tocsc()
    right = p.bc_nodes[p.bc_values == 0.0]
    left = p.bc_nodes[p.bc_values == 1.0]
    # some columns of the second boundary type survive, all of the first are gone
    kept = [c for c in right if np.count_nonzero(M[:, c].toarray().ravel()) > 1]
    assert len(kept) > 0
    assert all(np.count_nonzero(M[:, c].toarray().ravel()) == 1 for c in left)


def test_duplicate_dirichlet_last_value_wins(port, ref):
    p = meshgen.cube_scalar(n=4, n_spheres=0)
    nodes = np.concatenate([p.bc_nodes, p.bc_nodes[:3]])
    vals = np.concatenate([p.bc_values, [7.0, 8.0, 9.0]])
    p.bc_nodes, p.bc_values = nodes.astype(np.int32), vals
    A, _ = ref.scalar_system(p, stage=1)
    B = port.scalar_system(p, stage=1)
    _same_pattern(A, B)
    np.testing.assert_allclose(B.F, A.F, rtol=0, atol=1e-14)
    np.testing.assert_allclose(B.val, A.val, rtol=0, atol=1e-13)


def test_solvers_reproduce_reference_iterates(port, ref):
    p = meshgen.cube_elastic(n=4)
    A, _ = ref.elastic_system(p, stage=1)
    # MSG, MSG_PreconditioningSSOR(0.75), BiCG_Stab: bit-identical solutions
    for method, fn in ((0, port.cg), (1, port.pcg_ssor), (2, port.bicgstab)):
        xr, rr, _ = ref.cssd_solve(method, A, tol=1e-10)
        xp, rp, _ = fn(A, tol=1e-10)
        np.testing.assert_array_equal(xp, xr)
        assert rp == rr
    # GMRES(5) with its in-place row scaling, for 1..4 restarts
    for cycles in (1, 2, 4):
        xr, rr, _ = ref.cssd_solve(4, A, maxiter=cycles, tol=1e-10)
        xp, rp, _ = port.gmres_ref(A, maxiter=cycles, tol=1e-10)
        np.testing.assert_array_equal(xp, xr)


def test_ssor_preconditioner_matches_reference(port, ref):
    p = meshgen.cube_scalar(n=5, n_spheres=2, rmin=0.1, rmax=0.2)
    A, _ = ref.scalar_system(p, stage=1)
    r = np.random.default_rng(1).normal(size=A.n)
    np.testing.assert_array_equal(port.ssor_apply(A, r), ref.ssor_apply(A, r))


def test_restarted_gmres_and_jacobi_pcg_converge(port, ref):
    p = meshgen.cube_scalar(n=6, n_spheres=3, rmin=0.1, rmax=0.2)
    A, _ = ref.scalar_system(p, stage=1)
    xref, _, _ = ref.cssd_solve(0, A, tol=1e-13)
    for fn in (lambda: port.gmres(A, m=20, tol=1e-12), lambda: port.pcg_jacobi(A, tol=1e-12)):
        x, res, it = fn()
        assert res < 1e-11
        assert np.linalg.norm(x - xref) / np.linalg.norm(xref) < 1e-10


def test_reference_elasticity_matrix_is_symmetric_but_indefinite(port, ref):
    """The reference's transposed element blocks (FEM/FEM_Grid.h:2147-2191) keep the global
    elasticity matrix symmetric but make it indefinite (a null-Lagrangian term survives on
    couplings between free-boundary nodes).  This is why the GPU path offers MINRES and uses it
    inside the FP32 refinement for elasticity."""
    p = meshgen.cube_elastic(n=6, jitter=0.0)
    A, _ = ref.elastic_system(p, stage=1)
    M = A.to_scipy().toarray()
    assert np.abs(M - M.T).max() <= 1e-15 * np.abs(M).max()   # diagonal blocks: rounding only
    s = 1.0 / np.sqrt(np.diag(M))
    w = np.linalg.eigvalsh(s[:, None] * M * s[None, :])
    assert w[0] < -1e-3 and w[-1] > 1.0
