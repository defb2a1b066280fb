"""The FEM drivers' restart loop (FEM/FEM.h:627-695 for FEM_forBaseEliptic, :1853-1939 for
FEM_forElasticDeformation) restated around the C restatement's SSOR-PCG (oracle/port.py
driver_loop), against the reference's own drivers run here (oracle/_ref): the same solution bits."""
import numpy as np
import pytest

import oracle
from multiscalefemsolver3d_b200 import meshgen

needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("n,seed", [(4, 3), (6, 1)])
def test_elastic_loop_is_the_reference_driver(port, n, seed):
    R = oracle.ref()
    p = meshgen.cube_elastic(n=n, jitter=0.1, seed=seed)
    A, _ = R.elastic_system(p, stage=1)
    xr, _ = R.elastic_driver(p, min_residual=1e-10)
    x, best, log = port.driver_loop(A, 1, 1e-10)
    np.testing.assert_array_equal(x, xr)
    # targets tighten tenfold from 1e-2; the last solve (below 1e-10) is not the one returned
    assert log[0][0] == 1e-2 and log[-1][1] <= 1e-10 and best <= 1e-10


@needs_ref
@pytest.mark.parametrize("n", [5, 8])
def test_scalar_loop_is_the_reference_driver(port, n):
    R = oracle.ref()
    p = meshgen.cube_scalar(n=n, n_spheres=3, rmin=0.1, rmax=0.2)
    A, _ = R.scalar_system(p, stage=1)
    xr, _ = R.scalar_driver(p, min_residual=1e-10)
    x, best, log = port.driver_loop(A, 0, 1e-10)
    np.testing.assert_array_equal(x, xr)
    assert log[0][0] == 1e-1


def test_loop_returns_the_solution_before_the_last_solve(port):
    """The reference breaks out of its loop before copying the solve that reached MIN_RESIDUAL, so
    the loop's X is the best of the earlier solves: its residual lies above the last solve's."""
    p = meshgen.cube_scalar(n=6, n_spheres=2, rmin=0.1, rmax=0.2)
    A = port.scalar_system(p, stage=1)
    x, best, log = port.driver_loop(A, 0, 1e-9)
    r = A.F - A.to_scipy() @ x
    rel = np.linalg.norm(r) / np.linalg.norm(A.F)
    assert log[-1][1] <= 1e-9 < rel
