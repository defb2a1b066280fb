"""The allocation-free entry point, msfem_residual_noalloc, against the existing API.

It exists for callers that cannot let a library allocate device memory (an
application arena that owns the whole heap, or a loop that cannot take
cudaFree's device-wide synchronisation); its only scratch is a fixed device
array inside the library.  Here it is called twice in a row through the C ABI on
a caller-owned CSR copy of an assembled system, and each result is checked
against the residual built from the handle API's msfem_spmv.  This file is
collected last so that a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

from multiscalefemsolver3d_b200 import _lib, fem, meshgen

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the tolerance the parity tests use for assembled quantities


def test_noalloc_residual_matches_handle_api_twice(cuda):
    import torch
    p = meshgen.cube_scalar(n=14, n_spheres=10, rmin=0.05, rmax=0.1, contrast=100.0)
    L = _lib.load()
    with fem.System(fem.SCALAR, p.mesh.xyz, p.mesh.tets, p.mesh.mat) as S:
        S.assemble_scalar(p.sigma)
        S.apply_dirichlet(p.bc_nodes, p.bc_values, fem.ROW_AND_COLUMN)
        A = S.export_csr()
        rng = np.random.default_rng(7)
        dev = torch.device("cuda:0")
        rp = torch.from_numpy(A.row_ptr).to(dev)
        col = torch.from_numpy(A.col).to(dev)
        val = torch.from_numpy(A.val).to(dev)
        f = torch.from_numpy(A.F).to(dev)
        r = torch.empty(A.n, dtype=torch.float64, device=dev)
        rr = torch.empty(1, dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream(dev)
        P = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
        for call in range(2):
            xh = rng.normal(size=A.n)
            x = torch.from_numpy(xh).to(dev)
            torch.cuda.synchronize()
            rc = L.msfem_residual_noalloc(A.n, P(rp), P(col), P(val), P(x), P(f), P(r), P(rr),
                                          C.c_void_p(stream.cuda_stream))
            assert rc == 0, L.msfem_last_error()
            torch.cuda.synchronize()
            r_ref = A.F - S.spmv(xh)            # the existing entry point
            scale = np.abs(A.val).max() * np.abs(xh).max() * 15 + np.abs(A.F).max()
            np.testing.assert_allclose(r.cpu().numpy(), r_ref, rtol=0, atol=TOL * scale)
            rr_ref = float(r_ref @ r_ref)
            assert abs(rr.item() - rr_ref) <= TOL * rr_ref


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    import torch
    L = _lib.load()
    d = torch.zeros(4, dtype=torch.float64, device="cuda:0")
    i = torch.zeros(4, dtype=torch.int32, device="cuda:0")
    P = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    # the size check runs before any pointer is used
    rc = L.msfem_residual_noalloc(4_194_305, P(i), P(i), P(d), P(d), P(d), P(d), P(d), None)
    assert rc == _lib.MSFEM_ERR_LIMIT
    assert b"4194304" in L.msfem_last_error()


def _tridiagonal(n, seed):
    """CSR of a diagonally dominant tridiagonal matrix with n rows (row i: i-1, i, i+1)."""
    rng = np.random.default_rng(seed)
    counts = np.full(n, 3, np.int64)
    counts[0] = counts[-1] = 2
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(counts, out=rp[1:])
    rows = np.repeat(np.arange(n), counts)
    k = np.arange(rp[-1]) - rp[rows]
    col = (rows + k - (rows > 0)).astype(np.int32)
    val = np.where(col == rows, 4.0, -1.0) + rng.uniform(-0.1, 0.1, col.size)
    return rp.astype(np.int32), col, val


@pytest.mark.parametrize("sizes", [(600_000, 4_194_304, 1_000)])
def test_noalloc_large_grids_and_the_exact_limit(cuda, sizes):
    """A call of 600,000 rows (2,344 blocks: the 8-way unrolled partial sum), one of exactly
    4,194,304 rows (every slot of the fixed scratch), then a small call after the larger ones: r
    against the residual computed in numpy, ||r||^2 against its exactly rounded sum (math.fsum).
    The small call must not read partial sums the larger ones left in the shared array."""
    import math

    import torch
    L = _lib.load()
    dev = torch.device("cuda:0")
    P = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    stream = torch.cuda.current_stream(dev)
    for k, n in enumerate(sizes):
        rp, col, val = _tridiagonal(n, seed=k)
        rng = np.random.default_rng(100 + k)
        xh = rng.normal(size=n)
        fh = rng.normal(size=n)
        t = [torch.from_numpy(a).to(dev) for a in (rp, col, val, xh, fh)]
        r = torch.empty(n, dtype=torch.float64, device=dev)
        rr = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        rc = L.msfem_residual_noalloc(n, *[P(a) for a in t], P(r), P(rr), C.c_void_p(stream.cuda_stream))
        assert rc == 0, L.msfem_last_error()
        torch.cuda.synchronize()
        rows = np.repeat(np.arange(n), np.diff(rp))
        ax = np.bincount(rows, weights=val * xh[col], minlength=n)
        r_ref = fh - ax
        scale = np.abs(val).max() * np.abs(xh).max() * 3 + np.abs(fh).max()
        np.testing.assert_allclose(r.cpu().numpy(), r_ref, rtol=0, atol=TOL * scale)
        rr_ref = math.fsum((r_ref * r_ref).tolist())
        assert abs(rr.item() - rr_ref) <= TOL * rr_ref, (n, rr.item(), rr_ref)
        del t, r, rr
