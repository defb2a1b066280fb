"""The three-coefficient scalar FEM (stiffness + mass + source per element, FEM/FEM_Grid.h:25-102,
and its driver FEM_forBaseEliptic, FEM/FEM.h:206-397): the restatement oracle/scalar3.py against
the reference's own element and driver (oracle/_ref)."""
import numpy as np
import pytest

import oracle
from multiscalefemsolver3d_b200 import meshgen
from oracle import scalar3

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")


@needs_ref
def test_element_matches_reference():
    R = oracle.ref()
    rng = np.random.default_rng(3)
    for _ in range(20):
        P = rng.normal(size=(4, 3))
        S, M, f = rng.uniform(0.1, 10.0, 3)
        A, F = scalar3.local(P, S, M, f)
        Ar, Fr = R.scalar3_local(P, S, M, f)
        np.testing.assert_allclose(A, Ar, rtol=0, atol=1e-12 * np.abs(Ar).max())
        np.testing.assert_allclose(F, Fr, rtol=0, atol=1e-12 * np.abs(Fr).max())


@needs_ref
def test_driver_matches_reference():
    """6^3 jittered cube, per-element coefficients, u = 1 on x = 0 and 0 on x = 1 (rows only)."""
    R = oracle.ref()
    m = meshgen.kuhn_cube(6, jitter=0.1, seed=2)
    rng = np.random.default_rng(5)
    S = rng.uniform(0.5, 5.0, m.n_tets)
    M = rng.uniform(0.0, 2.0, m.n_tets)
    f = rng.uniform(-1.0, 1.0, m.n_tets)
    lo = np.nonzero(m.xyz[:, 0] < 1e-12)[0]
    hi = np.nonzero(m.xyz[:, 0] > 1 - 1e-12)[0]
    nodes = np.concatenate([lo, hi]).astype(np.int32)
    vals = np.concatenate([np.ones(lo.size), np.zeros(hi.size)])
    x = scalar3.driver(m.xyz, m.tets, S, M, f, nodes, vals)
    xr = R.scalar3_driver(m.xyz, m.tets, S, M, f, nodes, vals, min_residual=1e-13)
    assert np.linalg.norm(x - xr) <= 1e-9 * np.linalg.norm(xr)


def test_driver_orchestration_with_stand_in(monkeypatch, lib):
    """fem.fem_scalar3_driver end to end with its GPU system replaced by a stand-in that assembles
    with the restated element, applies rows-only Dirichlet data and solves exactly: the glue hands
    the coefficients, rows and solve through as the reference driver does."""
    from multiscalefemsolver3d_b200 import fem

    class FakeSystem:
        def __init__(self, kind, xyz, tets, material=None):
            assert kind == fem.SCALAR
            self.xyz, self.tets = np.asarray(xyz), np.asarray(tets)
            n = self.xyz.shape[0]
            self.A, self.F = np.zeros((n, n)), np.zeros(n)

        def assemble_scalar3(self, S, M, f):
            for e, t in enumerate(self.tets):
                A, Fe = scalar3.local(self.xyz[t], S[e], M[e], f[e])
                self.A[np.ix_(t, t)] += A
                self.F[t] += Fe

        def apply_dirichlet(self, dofs, values, mode):
            assert mode == fem.ROW_ONLY
            for i, v in zip(dofs, values):
                self.A[i, :] = 0.0
                self.A[i, i] = 1.0
                self.F[i] = v

        def solve(self, method, precision, tol, maxiter):
            assert method == fem.BICGSTAB and precision == fem.FP64
            self.x = np.linalg.solve(self.A, self.F)
            return 0.0, 1, 0

        def get_x(self):
            return self.x

        def close(self):
            pass

    monkeypatch.setattr(fem, "System", FakeSystem)
    m = meshgen.kuhn_cube(4, jitter=0.1, seed=6)
    rng = np.random.default_rng(8)
    S, M, f = rng.uniform(0.5, 3.0, m.n_tets), rng.uniform(0.0, 1.0, m.n_tets), rng.uniform(-1, 1, m.n_tets)
    lo = np.nonzero(m.xyz[:, 2] < 1e-12)[0].astype(np.int32)
    x, rel, it, rc = fem.fem_scalar3_driver(m.xyz, m.tets, S, M, f, lo, np.full(lo.size, 0.5))
    xo = scalar3.driver(m.xyz, m.tets, S, M, f, lo, np.full(lo.size, 0.5))
    assert rc == 0 and np.linalg.norm(x - xo) <= 1e-12 * np.linalg.norm(xo)
