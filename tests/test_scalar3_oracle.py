"""The three-coefficient scalar FEM (stiffness + mass + source per element, FEM/FEM_Grid.h:25-102,
and its driver FEM_forBaseEliptic, FEM/FEM.h:206-397): the restatement oracle/scalar3.py against
the reference's own element and driver (oracle/_ref)."""
import numpy as np
import pytest

import oracle
from multiscalefemsolver3d_b200 import meshgen
from oracle import scalar3

pytestmark = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")


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
