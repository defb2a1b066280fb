"""The three-coefficient scalar FEM on the GPU (FiniteElement_forScal::SolveLocalMatrix with
stiffness, mass and source coefficients, FEM/FEM_Grid.h:25-102, driven as FEM::FEM_forBaseEliptic
does at FEM/FEM.h:206-397) against oracle/scalar3.py, which tests/test_scalar3_oracle.py pins to
the reference's own element and driver.

Bars: pattern bit-exact (the node portrait), matrix values and F within 1e-12 of their largest
entries, the rows-only Dirichlet system exactly the reference's (identity rows, columns kept),
the BiCGStab driver's solution within 1e-8 relative L2 of the oracle's exact solve."""
import numpy as np
import pytest

from multiscalefemsolver3d_b200 import fem, meshgen
from oracle import scalar3

pytestmark = pytest.mark.gpu


def _case(n=8, seed=2):
    m = meshgen.kuhn_cube(n, jitter=0.1, seed=seed)
    rng = np.random.default_rng(seed + 3)
    S = rng.uniform(0.5, 5.0, m.n_tets)
    M = rng.uniform(0.0, 2.0, m.n_tets)
    f = rng.uniform(-1.0, 1.0, m.n_tets)
    return m, S, M, f


def _oracle_system(m, S, M, f, csr):
    """The restated element matrices summed into the GPU's CSR portrait (SummPartOfMatrix)."""
    val = np.zeros(csr.col.size)
    F = np.zeros(m.n_nodes)
    rp, col = csr.row_ptr, csr.col
    for e, t in enumerate(m.tets):
        A, Fe = scalar3.local(m.xyz[t], S[e], M[e], f[e])
        for i in range(4):
            row = col[rp[t[i]]:rp[t[i] + 1]]
            for j in range(4):
                val[rp[t[i]] + np.searchsorted(row, t[j])] += A[i, j]
        F[t] += Fe
    return val, F


def test_scalar3_assembly_matches_oracle(lib, cuda):
    m, S, M, f = _case()
    with fem.System(fem.SCALAR, m.xyz, m.tets) as G:
        G.assemble_scalar3(S, M, f)
        A = G.export_csr()
    # the node portrait: every pair of nodes of a tetrahedron couples, rows sorted, diagonal in place
    for i in range(m.n_nodes):
        assert np.all(np.diff(A.col[A.row_ptr[i]:A.row_ptr[i + 1]]) > 0)
    val, F = _oracle_system(m, S, M, f, A)
    assert np.abs(A.val - val).max() <= 1e-12 * np.abs(val).max()
    assert np.abs(A.F - F).max() <= 1e-12 * np.abs(F).max()
    # the mass term makes the matrix definite with a pure-Neumann boundary: all row sums = V M / 4
    assert np.all(A.to_scipy().sum(axis=1) > -1e-12)


def test_scalar3_rows_only_dirichlet_and_bicgstab_driver(lib, cuda):
    """u = 1 on x = 0 and 0 on x = 1 as identity rows (FEM.h:297-324): the system becomes
    nonsymmetric (the Dirichlet columns stay), the GPU BiCGStab solves it to 1e-12 and its solution
    matches the oracle driver's exact solve to 1e-8; the one-call driver gives the same."""
    m, S, M, f = _case(n=8, seed=4)
    lo = np.nonzero(m.xyz[:, 0] < 1e-12)[0]
    hi = np.nonzero(m.xyz[:, 0] > 1 - 1e-12)[0]
    nodes = np.concatenate([lo, hi, lo[:5]]).astype(np.int32)          # a repeated node: the later value wins
    vals = np.concatenate([np.ones(lo.size), np.zeros(hi.size), np.full(5, 1.0)])
    want = scalar3.driver(m.xyz, m.tets, S, M, f, nodes, vals)
    with fem.System(fem.SCALAR, m.xyz, m.tets) as G:
        G.assemble_scalar3(S, M, f)
        G.apply_dirichlet(nodes, vals, fem.ROW_ONLY)
        A = G.export_csr()
        K = A.to_scipy().tocsr()
        for v in np.unique(nodes):
            row = K.getrow(v)
            assert row.nnz >= 1 and row[0, v] == 1.0 and np.count_nonzero(row.toarray()) == 1
        assert abs(K - K.T).max() > 0                                   # rows only: not symmetric
        assert np.all(A.F[nodes[:lo.size]] == 1.0) and np.all(A.F[hi] == 0.0)
        rel, it, rc = G.solve(fem.BICGSTAB, fem.FP64, tol=1e-12, maxiter=20000)
        assert rc == 0 and rel <= 1e-12
        x = G.get_x()
    assert np.linalg.norm(x - want) <= 1e-8 * np.linalg.norm(want)
    x2, rel2, it2, rc2 = fem.fem_scalar3_driver(m.xyz, m.tets, S, M, f, nodes, vals, min_residual=1e-12)
    assert rc2 == 0 and np.linalg.norm(x2 - want) <= 1e-8 * np.linalg.norm(want)


def test_scalar3_device_coefficients_and_repeat(lib, cuda):
    """Coefficients handed in as device arrays give the same bits as host arrays, and two
    assemblies after a clear give the same bits (coloured, deterministic scatter)."""
    import ctypes as C

    import torch
    from multiscalefemsolver3d_b200 import _lib
    m, S, M, f = _case(n=6, seed=9)
    with fem.System(fem.SCALAR, m.xyz, m.tets) as G:
        G.assemble_scalar3(S, M, f)
        A1 = G.export_csr()
        G.clear()
        d = [torch.from_numpy(np.ascontiguousarray(a)).to(cuda) for a in (S, M, f)]
        rc = _lib.load().msfem_assemble_scalar3(G.h, *[C.c_void_p(t.data_ptr()) for t in d], 1)
        assert rc == 0
        A2 = G.export_csr()
    np.testing.assert_array_equal(A1.val, A2.val)
    np.testing.assert_array_equal(A1.F, A2.F)
