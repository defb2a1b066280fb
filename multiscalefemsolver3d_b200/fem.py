"""Python view of the C ABI: one `System` per assembled matrix, plus the two
driver calls.  Method names follow the reference's step names
(CreationPortrait -> System(...), SolveLocalMatrix + SummPartOfMatrix ->
assemble_*, first/second boundary conditions -> apply_dirichlet /
add_traction, MSG / MSG_PreconditioningSSOR -> solve).

Arrays may be numpy arrays (host) or torch CUDA tensors (device, used in
place).  Every call goes through libmsfem_b200.so; nothing here computes.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import (BICGSTAB, CG, ELASTIC, FP32_IR, FP64, FP64_REFERENCE, GMRES, LOOP_ELASTIC, LOOP_SCALAR, MINRES, PCG_JACOBI, PCG_SSOR,
                   ROW_AND_COLUMN, ROW_ONLY, SCALAR, Stats, check, load)

__all__ = ["System", "Csr", "fem_scalar_driver", "fem_scalar3_driver", "fem_elastic_driver", "CG", "PCG_JACOBI",
           "BICGSTAB", "GMRES", "MINRES", "PCG_SSOR", "LOOP_SCALAR", "LOOP_ELASTIC", "FP64", "FP32_IR", "FP64_REFERENCE", "ROW_ONLY",
           "ROW_AND_COLUMN", "SCALAR", "ELASTIC"]


def _ptr(a, dtype):
    """(pointer, on_device, keepalive) for a numpy array or a torch tensor."""
    if a is None:
        return None, 0, None
    if hasattr(a, "data_ptr") and hasattr(a, "is_cuda"):
        if a.is_cuda:
            import torch
            want = {np.float64: torch.float64, np.int32: torch.int32, np.float32: torch.float32}[dtype]
            if a.dtype != want or not a.is_contiguous():
                raise TypeError(f"device tensor must be contiguous {want}")
            return C.c_void_p(a.data_ptr()), 1, a
        a = a.cpu().numpy()
    arr = np.ascontiguousarray(a, dtype=dtype)
    return arr.ctypes.data_as(C.c_void_p), 0, arr


@dataclass
class Csr:
    """CSR with the diagonal in place; row = reference CSSD row [A_down | Diag | A_up]."""
    row_ptr: np.ndarray
    col: np.ndarray
    val: np.ndarray
    F: np.ndarray
    X: np.ndarray

    @property
    def n(self) -> int:
        return self.row_ptr.size - 1

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.val, self.col, self.row_ptr), shape=(self.n, self.n))

    def cssd(self):
        """(Diag, A_up, A_down, id_column_for_A_up, id_column_for_A_down) as in Library/CSSD_Matrix.h:11-13."""
        diag = np.zeros(self.n)
        up, down, cu, cd = [], [], [], []
        for i in range(self.n):
            c = self.col[self.row_ptr[i]:self.row_ptr[i + 1]]
            v = self.val[self.row_ptr[i]:self.row_ptr[i + 1]]
            d = np.searchsorted(c, i)
            diag[i] = v[d]
            down.append(v[:d]); cd.append(c[:d])
            up.append(v[d + 1:]); cu.append(c[d + 1:])
        return diag, up, down, cu, cd


class System:
    """An assembled FEM system on the GPU (Grid + CSSD_Matrix of the reference)."""

    def __init__(self, kind: int, xyz, tets, material=None):
        L = load()
        self.kind = kind
        px, dx, kx = _ptr(xyz, np.float64)
        pt, dt, kt = _ptr(tets, np.int32)
        pm, dm, km = _ptr(material, np.int32)
        n_nodes = int(xyz.shape[0]) if xyz.ndim == 2 else int(xyz.shape[0] // 3)
        n_tets = int(tets.shape[0]) if tets.ndim == 2 else int(tets.shape[0] // 4)
        h = C.c_void_p()
        check(L.msfem_system_create(kind, n_nodes, px, n_tets, pt, pm, int(dx or dt), C.byref(h)), "system_create")
        self.h = h
        self.n_nodes = n_nodes
        self.n_tets = n_tets
        n_rows, nnz, nc = C.c_int(), C.c_int64(), C.c_int()
        check(L.msfem_system_info(h, C.byref(n_rows), C.byref(nnz), C.byref(nc)), "system_info")
        self.n_rows, self.nnz, self.n_colors = n_rows.value, nnz.value, nc.value

    @classmethod
    def from_cssd(cls, diag, down_cols, down_vals, up_cols, up_vals, F=None, X=None):
        """A scalar system from the reference's CSSD_Matrix arrays (per row i: A_down[i] with
        id_column_for_A_down[i], Diag[i], A_up[i] with id_column_for_A_up[i]); no mesh."""
        L = load()
        diag = np.ascontiguousarray(diag, dtype=np.float64)
        n = diag.size

        def flat(cols, vals):
            ptr = np.zeros(n + 1, np.int64)
            ptr[1:] = np.cumsum([len(c) for c in cols])
            c = np.ascontiguousarray(np.concatenate([np.asarray(x, np.int32) for x in cols]) if ptr[-1] else
                                     np.zeros(1, np.int32), dtype=np.int32)
            v = np.ascontiguousarray(np.concatenate([np.asarray(x, np.float64) for x in vals]) if ptr[-1] else
                                     np.zeros(1), dtype=np.float64)
            return ptr, c, v

        dp, dc, dv = flat(down_cols, down_vals)
        up, uc, uv = flat(up_cols, up_vals)
        keep = [diag, dp, dc, dv, up, uc, uv]
        Fa = None if F is None else np.ascontiguousarray(F, dtype=np.float64)
        Xa = None if X is None else np.ascontiguousarray(X, dtype=np.float64)
        P = lambda a: None if a is None else a.ctypes.data_as(C.c_void_p)  # noqa: E731
        h = C.c_void_p()
        check(L.msfem_system_from_cssd(n, P(diag), P(dp), P(dc), P(dv), P(up), P(uc), P(uv), P(Fa), P(Xa), C.byref(h)),
              "system_from_cssd")
        del keep
        return cls._from_handle(h)

    @classmethod
    def _from_handle(cls, h):
        """Wraps a scalar matrix-only system handle (no mesh)."""
        self = cls.__new__(cls)
        self.kind = SCALAR
        self.h = h
        self.n_tets = 0
        n_rows, nnz, nc = C.c_int(), C.c_int64(), C.c_int()
        check(load().msfem_system_info(h, C.byref(n_rows), C.byref(nnz), C.byref(nc)), "system_info")
        self.n_rows, self.nnz, self.n_colors = n_rows.value, nnz.value, nc.value
        self.n_nodes = self.n_rows
        return self

    @classmethod
    def from_csr(cls, A, F=None, X=None):
        """A scalar system from a Csr (diagonal present in every row), split into the CSSD parts."""
        diag, up, down, cu, cd = A.cssd()
        return cls.from_cssd(diag, cd, down, cu, up, F, X)

    def close(self):
        if getattr(self, "h", None):
            load().msfem_system_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- assembly and boundary conditions
    def assemble_scalar(self, sigma):
        s = np.ascontiguousarray(sigma, dtype=np.float64)
        check(load().msfem_assemble_scalar(self.h, s.ctypes.data_as(C.c_void_p), s.size), "assemble_scalar")

    def assemble_scalar3(self, S, M, f):
        """The three-coefficient element (stiffness S, mass M, source f per tetrahedron, at its
        centroid): A += V (S grad.grad + M / 16), F += V f / 4 (msfem_assemble_scalar3)."""
        a = [np.ascontiguousarray(np.broadcast_to(np.asarray(x, dtype=np.float64), (self.n_tets,))) for x in (S, M, f)]
        check(load().msfem_assemble_scalar3(self.h, *[x.ctypes.data_as(C.c_void_p) for x in a], 0), "assemble_scalar3")

    def assemble_elastic(self, E, nu):
        e = np.ascontiguousarray(E, dtype=np.float64)
        n = np.ascontiguousarray(nu, dtype=np.float64)
        check(load().msfem_assemble_elastic(self.h, e.ctypes.data_as(C.c_void_p), n.ctypes.data_as(C.c_void_p),
                                            e.size), "assemble_elastic")

    def assemble_elastic_textbook(self, E, nu):
        """The transposed (textbook, SPD) orientation of every element block; for preconditioners."""
        e = np.ascontiguousarray(E, dtype=np.float64)
        n = np.ascontiguousarray(nu, dtype=np.float64)
        check(load().msfem_assemble_elastic_textbook(self.h, e.ctypes.data_as(C.c_void_p),
                                                     n.ctypes.data_as(C.c_void_p), e.size), "assemble_elastic_textbook")

    def add_traction(self, faces, traction):
        pf, d1, k1 = _ptr(faces, np.int32)
        pt, d2, k2 = _ptr(traction, np.float64)
        nf = int(faces.shape[0]) if faces.ndim == 2 else int(faces.shape[0] // 3)
        check(load().msfem_add_traction(self.h, nf, pf, pt, int(d1 or d2)), "add_traction")

    def add_rhs(self, f):
        p, d, k = _ptr(f, np.float64)
        check(load().msfem_add_rhs(self.h, p, d), "add_rhs")

    def apply_dirichlet(self, dofs, values, mode: int = ROW_AND_COLUMN):
        pd, d1, k1 = _ptr(dofs, np.int32)
        pv, d2, k2 = _ptr(values, np.float64)
        n = int(np.asarray(dofs.shape).prod()) if hasattr(dofs, "shape") else len(dofs)
        check(load().msfem_apply_dirichlet(self.h, n, pd, pv, mode, int(d1 or d2)), "apply_dirichlet")

    def clear(self):
        check(load().msfem_clear(self.h), "clear")

    # -- vectors
    def set_x(self, x):
        p, d, k = _ptr(x, np.float64)
        check(load().msfem_set_x(self.h, p, d), "set_x")

    def get_x(self, out=None):
        out = np.empty(self.n_rows) if out is None else out
        p, d, k = _ptr(out, np.float64)
        check(load().msfem_get_x(self.h, p, d), "get_x")
        return out

    def postprocess_elastic(self, E, nu):
        """[n_tets, 23] per tetrahedron at its centroid from the current X: U, grad U (row a =
        grad u_a), sigma (xx yy zz yz xz xy, the element's material), von Mises, and the
        reference driver's printed sigma_xx, sigma_yy, sigma_zz, von Mises (domain 0's material)."""
        E = np.ascontiguousarray(E, dtype=np.float64)
        nu = np.ascontiguousarray(nu, dtype=np.float64)
        out = np.empty((self.n_tets, 23))
        check(load().msfem_postprocess_elastic(self.h, E.size, E.ctypes.data_as(C.c_void_p),
                                               nu.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p), 0),
              "postprocess_elastic")
        return out

    def get_f(self):
        out = np.empty(self.n_rows)
        check(load().msfem_get_f(self.h, out.ctypes.data_as(C.c_void_p), 0), "get_f")
        return out

    def copy_f_to_x(self):
        check(load().msfem_copy_f_to_x(self.h), "copy_f_to_x")

    # -- solve
    def solve(self, method: int = PCG_JACOBI, precision: int = FP64, tol: float = 1e-10, maxiter: int = 100000,
              restart: int = 30):
        rel, it = C.c_double(), C.c_int()
        rc = check(load().msfem_solve(self.h, method, precision, restart, maxiter, tol, C.byref(rel), C.byref(it)),
                   "solve")
        return rel.value, it.value, rc

    def set_ssor_omega(self, omega: float):
        """The relaxation factor of PCG_SSOR (PrecondorSSOR(omega, ...); default 0.75)."""
        check(load().msfem_set_ssor_omega(self.h, float(omega)), "set_ssor_omega")

    def ssor_apply(self, r):
        """z = M^-1 r with the reference's SSOR (SolvePrecondorSSOR_SLAE) on the current matrix."""
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.empty(self.n_rows)
        check(load().msfem_ssor_apply(self.h, r.ctypes.data_as(C.c_void_p), z.ctypes.data_as(C.c_void_p), 0),
              "ssor_apply")
        return z

    def solve_driver_loop(self, loop: int, method: int = PCG_SSOR, precision: int = FP64,
                          min_residual: float = 1e-10):
        """The reference driver's restart loop around `method` (LOOP_SCALAR: FEM_forBaseEliptic, which
        sets X = F first; LOOP_ELASTIC: FEM_forElasticDeformation); X ends as the loop's best
        solution.  Returns (best_residual, n_solves, total_iterations)."""
        best, ns, it = C.c_double(), C.c_int(), C.c_int()
        check(load().msfem_solve_driver_loop(self.h, loop, method, precision, min_residual, C.byref(best),
                                             C.byref(ns), C.byref(it)), "solve_driver_loop")
        return best.value, ns.value, it.value

    def spmv(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.n_rows)
        check(load().msfem_spmv(self.h, x.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p), 0), "spmv")
        return y

    def spmv_scaled32(self, x):
        """y = D^-1/2 A D^-1/2 x in FP32 (the operator of the FP32 inner solves)."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.empty(self.n_rows, dtype=np.float32)
        check(load().msfem_spmv_scaled32(self.h, x.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p), 0),
              "spmv_scaled32")
        return y

    def set_kuhn_grid(self, nx, ny=None, nz=None):
        """Declares the mesh a structured Kuhn grid of nx x ny x nz hexahedra (the layout of
        meshgen.kuhn_cube); checked on the device, MsfemError if the mesh is not that grid."""
        ny = nx if ny is None else ny
        nz = nx if nz is None else nz
        check(load().msfem_set_kuhn_grid(self.h, int(nx), int(ny), int(nz)), "set_kuhn_grid")

    def kuhn_spmv(self, x):
        """y = A x formed matrix-free on the Kuhn grid from the tetrahedra's materials (FP64)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty(self.n_rows)
        check(load().msfem_kuhn_spmv(self.h, x.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p), 0),
              "kuhn_spmv")
        return y

    def kuhn_spmv_scaled32(self, x):
        """y = S A S x in FP32 formed matrix-free on the Kuhn grid by the smoother's kernel (input
        scaled and masked first); S as spmv_scaled32's."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.empty(self.n_rows, dtype=np.float32)
        check(load().msfem_kuhn_spmv_scaled32(self.h, x.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p), 0),
              "kuhn_spmv_scaled32")
        return y

    def export_csr(self) -> Csr:
        rp = np.empty(self.n_rows + 1, dtype=np.int32)
        col = np.empty(self.nnz, dtype=np.int32)
        val = np.empty(self.nnz)
        check(load().msfem_export_csr(self.h, rp.ctypes.data_as(C.c_void_p), col.ctypes.data_as(C.c_void_p),
                                      val.ctypes.data_as(C.c_void_p), 0), "export_csr")
        return Csr(rp, col, val, self.get_f(), self.get_x())

    def stats(self) -> dict:
        st = Stats()
        check(load().msfem_get_stats(self.h, C.byref(st)), "get_stats")
        return st.as_dict()

    def bench_spmv(self, precision: int = FP64, reps: int = 50):
        ms, nb = C.c_double(), C.c_int64()
        check(load().msfem_bench_spmv(self.h, precision, reps, C.byref(ms), C.byref(nb)), "bench_spmv")
        return ms.value, nb.value

    @property
    def stream(self) -> int:
        return load().msfem_get_stream(self.h) or 0


# ------------------------------------------------------------------ one-call drivers

def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def fem_scalar_driver(p, method=PCG_JACOBI, precision=FP64, min_residual=1e-10, maxiter=200000):
    """FEM::FEM_forBaseEliptic (stiffness-only) on the GPU; returns (solution, stats, rc)."""
    m = p.mesh
    xyz, tets, mat = _c(m.xyz, np.float64), _c(m.tets, np.int32), _c(m.mat, np.int32)
    sig, bn, bv = _c(p.sigma, np.float64), _c(p.bc_nodes, np.int32), _c(p.bc_values, np.float64)
    sol = np.empty(m.n_nodes)
    st = Stats()
    P = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    rc = check(load().msfem_fem_scalar_driver(m.n_nodes, P(xyz), m.n_tets, P(tets), P(mat), sig.size, P(sig),
                                               bn.size, P(bn), P(bv), method, precision, min_residual, maxiter,
                                               P(sol), C.byref(st)), "fem_scalar_driver")
    return sol, st.as_dict(), rc


def fem_elastic_driver(p, method=PCG_JACOBI, precision=FP64, min_residual=1e-10, maxiter=200000):
    """FEM::FEM_forElasticDeformation on the GPU; returns (solution[3n], stats, rc)."""
    m = p.mesh
    xyz, tets, mat = _c(m.xyz, np.float64), _c(m.tets, np.int32), _c(m.mat, np.int32)
    E, nu = _c(p.E, np.float64), _c(p.nu, np.float64)
    bn, bm, bv = _c(p.bc_nodes, np.int32), _c(p.bc_mask, np.int32), _c(p.bc_values, np.float64)
    fc, ft = _c(p.faces, np.int32), _c(p.traction, np.float64)
    sol = np.empty(3 * m.n_nodes)
    st = Stats()
    P = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    rc = check(load().msfem_fem_elastic_driver(m.n_nodes, P(xyz), m.n_tets, P(tets), P(mat), E.size, P(E), P(nu),
                                                bn.size, P(bn), P(bm), P(bv), fc.shape[0], P(fc), P(ft), method,
                                                precision, min_residual, maxiter, P(sol), C.byref(st)),
               "fem_elastic_driver")
    return sol, st.as_dict(), rc


def fem_scalar3_driver(xyz, tets, S, M, f, bc_nodes, bc_values, min_residual=1e-10, maxiter=200000):
    """The three-coefficient FEM::FEM_forBaseEliptic (FEM/FEM.h:206-397) on the GPU: the element loop
    with stiffness, mass and source coefficients per tetrahedron (msfem_assemble_scalar3), Dirichlet
    rows only (X = F = value, the columns left, FEM.h:291-310; later duplicates win), BiCGStab in
    FP64 to ||F - A x|| <= min_residual ||F||.  Returns (solution, rel_residual, iterations, rc)."""
    S_ = System(SCALAR, np.asarray(xyz, dtype=np.float64), np.asarray(tets, dtype=np.int32))
    try:
        S_.assemble_scalar3(S, M, f)
        S_.apply_dirichlet(np.asarray(bc_nodes, dtype=np.int32), np.asarray(bc_values, dtype=np.float64), ROW_ONLY)
        rel, it, rc = S_.solve(BICGSTAB, FP64, tol=min_residual, maxiter=maxiter)
        return S_.get_x(), rel, it, rc
    finally:
        S_.close()
