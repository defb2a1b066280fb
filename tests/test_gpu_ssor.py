"""The reference's SSOR preconditioner, its PCG and the drivers' restart loop on the GPU
(CSSD_Matrix::PrecondorSSOR + SolvePrecondorSSOR_SLAE, Library/CSSD_Matrix.h:458-547;
MSG_PreconditioningSSOR, :1302-1398; FEM/FEM.h:627-695, :1853-1939) against the C restatement
(oracle/femoracle.c, whose SSOR and PCG give the reference's bits, tests/test_oracle.py) and the
restated loop (oracle/port.py driver_loop, which returns the reference drivers' own bits,
tests/test_driver_loop_oracle.py).

Bars: one SSOR application bit-identical to the restatement (the level-scheduled sweeps repeat each
row's operations in the reference's order, unfused).  With precision FP64_REFERENCE (the reference's
operation order everywhere: serial inner products, the CSSD row order of A x, unfused updates) the
SSOR-PCG and the whole restart loop give the restatement's bits -- iterates, iteration counts and
returned residuals.  With the default FP64 (tree-summed inner products) the SSOR-PCG iteration count
stays within 2 of the restatement's on one solve and its solution within 1e-8; across the restart
loop, whose solves stop at loose tolerances where CG's residual oscillates, the rounding of the
inner products moves each solve's stopping iteration, so there only the solve count and the
solution (1e-8) are compared.
"""
import os

import numpy as np
import pytest

from multiscalefemsolver3d_b200 import fem, meshgen

pytestmark = pytest.mark.gpu
G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _elastic(n=6, spheres=3, seed=2):
    p = meshgen.cube_elastic(n=n, jitter=0.1, seed=seed, n_spheres=spheres, contrast=20.0, rmin=0.1, rmax=0.2)
    S = fem.System(fem.ELASTIC, p.mesh.xyz, p.mesh.tets, p.mesh.mat)
    S.add_traction(p.faces, p.traction)
    S.assemble_elastic(p.E, p.nu)
    dofs = (3 * p.bc_nodes[:, None] + np.arange(3)).ravel().astype(np.int32)
    S.apply_dirichlet(dofs, np.ascontiguousarray(p.bc_values.ravel()), fem.ROW_AND_COLUMN)
    return p, S


def _scalar(n=8, spheres=4):
    p = meshgen.cube_scalar(n=n, n_spheres=spheres, rmin=0.1, rmax=0.2, contrast=100.0)
    S = fem.System(fem.SCALAR, p.mesh.xyz, p.mesh.tets, p.mesh.mat)
    S.assemble_scalar(p.sigma)
    S.apply_dirichlet(p.bc_nodes, p.bc_values, fem.ROW_AND_COLUMN)
    return p, S


@pytest.mark.parametrize("kind", ["scalar", "elastic"])
@pytest.mark.parametrize("w", [0.75, 1.3])
def test_ssor_application_is_bit_identical(lib, cuda, port, kind, w):
    p, S = _scalar() if kind == "scalar" else _elastic()
    with S:
        A = S.export_csr()
        S.set_ssor_omega(w)
        for seed in range(2):
            r = np.random.default_rng(seed).normal(size=A.n)
            np.testing.assert_array_equal(S.ssor_apply(r), port.ssor_apply(A, r, w=w))


@pytest.mark.parametrize("kind", ["scalar", "elastic"])
def test_pcg_ssor_follows_the_restatement(lib, cuda, port, kind):
    """The default order on one solve to 1e-12: on the SPD scalar system the iteration count stays
    within 2 of the restatement's; on the reference's indefinite elasticity matrix CG's count is
    sensitive to the rounding of the inner products (1,054 against 1,120 measured on this 6^3 case),
    so there only the solution is compared."""
    p, S = _scalar() if kind == "scalar" else _elastic()
    with S:
        A = S.export_csr()
        S.set_x(np.zeros(A.n))
        rel, it, rc = S.solve(fem.PCG_SSOR, fem.FP64, tol=1e-12, maxiter=10000)
        x = S.get_x()
    xo, res_o, it_o = port.pcg_ssor(A, X0=np.zeros(A.n), maxiter=10001, tol=1e-12)
    # the stop is on the recurrence residual; the true one (reported) drifts a little above it
    assert rc == 0 and rel <= 1e-11
    if kind == "scalar":
        assert abs(it - it_o) <= 2, (it, it_o)
    assert np.linalg.norm(x - xo) <= 1e-8 * np.linalg.norm(xo)


@pytest.mark.parametrize("kind", ["scalar", "elastic"])
@pytest.mark.parametrize("tol", [1e-4, 1e-12])
def test_pcg_ssor_reference_order_is_bit_identical(lib, cuda, port, kind, tol):
    """MSG_PreconditioningSSOR in the reference's operation order: the restatement's iterate, its
    iteration count and its returned residual, bit for bit (maxiter = 10,001 there: its loop runs
    while k < maxiter, at most 10,000 iterations)."""
    p, S = _scalar() if kind == "scalar" else _elastic()
    with S:
        A = S.export_csr()
        S.set_x(np.zeros(A.n))
        rel, it, rc = S.solve(fem.PCG_SSOR, fem.FP64_REFERENCE, tol=tol, maxiter=10000)
        x = S.get_x()
    xo, res_o, it_o = port.pcg_ssor(A, X0=np.zeros(A.n), maxiter=10001, tol=tol)
    assert it == it_o, (it, it_o)
    np.testing.assert_array_equal(x, xo)
    assert rel == res_o, (rel, res_o)


def test_pcg_ssor_rejects_fp32(lib, cuda):
    from multiscalefemsolver3d_b200 import _lib
    p, S = _scalar(n=4, spheres=1)
    with S:
        with pytest.raises(_lib.MsfemError) as e:
            S.solve(fem.PCG_SSOR, fem.FP32_IR, tol=1e-8)
        assert e.value.rc == _lib.MSFEM_ERR_ARGUMENT


@pytest.mark.parametrize("loop", [fem.LOOP_SCALAR, fem.LOOP_ELASTIC])
def test_driver_loop_reference_order_is_bit_identical(lib, cuda, port, loop):
    """The restart loop on the GPU in the reference's operation order against the restated loop on
    the same matrix (whose bits are the reference driver's, tests/test_driver_loop_oracle.py): the
    same solves, the same iterations, the same returned solution bits."""
    p, S = _scalar() if loop == fem.LOOP_SCALAR else _elastic()
    with S:
        A = S.export_csr()
        best, n_solves, its = S.solve_driver_loop(loop, fem.PCG_SSOR, fem.FP64_REFERENCE, min_residual=1e-10)
        x = S.get_x()
    xo, best_o, log = port.driver_loop(A, loop, 1e-10)
    assert n_solves == len(log), (n_solves, len(log))
    assert its == sum(e[2] for e in log), (its, [e[2] for e in log])
    assert best == best_o
    np.testing.assert_array_equal(x, xo)


@pytest.mark.parametrize("loop", [fem.LOOP_SCALAR, fem.LOOP_ELASTIC])
def test_driver_loop_fast_order_follows_the_restated_loop(lib, cuda, port, loop):
    """The default (tree-summed) order: the same solve count, and a returned solution as close to
    the exact one as the restated loop's (both stop near 1e-10 in the residual; which iterate each
    returns depends on the stopping iterations).  The iteration total is not compared (see the
    module docstring)."""
    import scipy.sparse.linalg as spl
    p, S = _scalar() if loop == fem.LOOP_SCALAR else _elastic()
    with S:
        A = S.export_csr()
        best, n_solves, its = S.solve_driver_loop(loop, fem.PCG_SSOR, fem.FP64, min_residual=1e-10)
        x = S.get_x()
    xo, best_o, log = port.driver_loop(A, loop, 1e-10)
    assert n_solves == len(log), (n_solves, len(log))
    assert best <= 1e-10 and best_o <= 1e-10
    xe = spl.spsolve(A.to_scipy().tocsc(), A.F)
    err, err_o = np.linalg.norm(x - xe), np.linalg.norm(xo - xe)
    assert err <= max(10 * err_o, 1e-9 * np.linalg.norm(xe)), (err, err_o)


def test_c1_elastic_driver_with_the_reference_solve(lib, cuda):
    """FEM_forElasticDeformation on the full 20^3 workload with the reference's own solve (SSOR(0.75)
    -PCG in its restart loop) through the one-call driver: within 1e-8 of the reference driver's
    output (tests/golden/c1_elastic.npz, x_driver) and of its tight CG solution (x_cg)."""
    d = np.load(os.path.join(G, "c1_elastic.npz"))
    p = meshgen.cube_elastic(n=int(d["n"]), jitter=float(d["jitter"]), seed=int(d["seed"]))
    x, stats, rc = fem.fem_elastic_driver(p, method=fem.PCG_SSOR, precision=fem.FP64_REFERENCE,
                                          min_residual=1e-10)
    assert rc == 0
    for key in ("x_driver", "x_cg"):
        xr = d[key]
        assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-8, key


def test_scalar_driver_with_the_reference_solve(lib, cuda, port):
    """FEM_forBaseEliptic through the one-call driver with the reference's own solve: within 1e-8 of
    the restated loop on the restated system (the loop's bits are the reference driver's)."""
    p = meshgen.cube_scalar(n=10, n_spheres=5, rmin=0.08, rmax=0.15, contrast=100.0)
    for precision in (fem.FP64, fem.FP64_REFERENCE):
        x, stats, rc = fem.fem_scalar_driver(p, method=fem.PCG_SSOR, precision=precision, min_residual=1e-10)
        assert rc == 0
        A = port.scalar_system(p, stage=1)
        xo, best, log = port.driver_loop(A, 0, 1e-10)
        assert np.linalg.norm(x - xo) <= 1e-8 * np.linalg.norm(xo)
