"""Test infrastructure only: ctypes bindings of the C restatement (femoracle.c)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "_build", "libfemoracle.so")

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


class _FoCsr(C.Structure):
    _fields_ = [("n", C.c_int), ("nnz", C.c_longlong), ("row_ptr", C.POINTER(C.c_int)),
                ("col", C.POINTER(C.c_int)), ("val", C.POINTER(C.c_double)),
                ("F", C.POINTER(C.c_double)), ("X", C.POINTER(C.c_double))]


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


class PortLib:
    def __init__(self, path: str = PORT_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: build it with `make -C oracle oracle`")
        L = C.CDLL(path)
        self.L = L
        L.fo_free_csr.argtypes = [C.POINTER(_FoCsr)]
        L.fo_elastic_local.argtypes = [_f64p, C.c_double, C.c_double, _f64p]
        L.fo_scalar_local.argtypes = [_f64p, C.c_double, _f64p]
        mesh = [C.c_int, _f64p, C.c_int, _i32p, _i32p]
        L.fo_elastic_system.argtypes = mesh + [C.c_int, _f64p, _f64p, C.c_int, _i32p, _i32p, _f64p,
                                               C.c_int, _i32p, _i32p, _f64p, C.c_int, C.POINTER(_FoCsr)]
        L.fo_scalar_system.argtypes = mesh + [C.c_int, _f64p, C.c_int, _i32p, _f64p, C.c_int, C.POINTER(_FoCsr)]
        L.fo_spmv.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p]
        sol = [C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p]
        L.fo_cg.argtypes = sol + [C.c_int, C.c_double, C.POINTER(C.c_int)]
        L.fo_pcg_ssor.argtypes = sol + [C.c_int, C.c_double, C.c_double, C.POINTER(C.c_int)]
        L.fo_pcg_jacobi.argtypes = sol + [C.c_int, C.c_double, C.POINTER(C.c_int)]
        L.fo_bicgstab.argtypes = sol + [C.c_int, C.c_double, C.POINTER(C.c_int)]
        L.fo_gmres.argtypes = sol + [C.c_int, C.c_int, C.c_double, C.POINTER(C.c_int)]
        L.fo_gmres_ref.argtypes = sol + [C.c_int, C.c_double, C.POINTER(C.c_int)]
        L.fo_ssor_apply.argtypes = [C.c_int, _i32p, _i32p, _f64p, C.c_double, _f64p, _f64p]
        L.fo_minres.argtypes = sol + [C.c_int, C.c_double, C.POINTER(C.c_int)]
        for f in ("fo_cg", "fo_pcg_ssor", "fo_pcg_jacobi", "fo_bicgstab", "fo_gmres", "fo_gmres_ref", "fo_minres"):
            getattr(L, f).restype = C.c_double

    @staticmethod
    def _take(out):
        from . import Csr
        n, nnz = out.n, out.nnz
        return Csr(
            row_ptr=np.ctypeslib.as_array(out.row_ptr, shape=(n + 1,)).copy(),
            col=np.ctypeslib.as_array(out.col, shape=(nnz,)).copy(),
            val=np.ctypeslib.as_array(out.val, shape=(nnz,)).copy(),
            F=np.ctypeslib.as_array(out.F, shape=(n,)).copy(),
            X=np.ctypeslib.as_array(out.X, shape=(n,)).copy(),
        )

    def elastic_local(self, xyz4, E=1.0, nu=0.3):
        K = np.zeros(144)
        self.L.fo_elastic_local(_c(xyz4, np.float64).ravel(), E, nu, K)
        return K.reshape(4, 4, 3, 3)

    def scalar_local(self, xyz4, sigma=1.0):
        K = np.zeros(16)
        self.L.fo_scalar_local(_c(xyz4, np.float64).ravel(), sigma, K)
        return K.reshape(4, 4)

    def elastic_system(self, p, stage: int = 1):
        m = p.mesh
        out = _FoCsr()
        self.L.fo_elastic_system(
            m.n_nodes, _c(m.xyz, np.float64).ravel(), m.n_tets, _c(m.tets, np.int32).ravel(), _c(m.mat, np.int32),
            len(p.E), _c(p.E, np.float64), _c(p.nu, np.float64),
            len(p.bc_nodes), _c(p.bc_nodes, np.int32), _c(p.bc_mask, np.int32), _c(p.bc_values, np.float64).ravel(),
            len(p.face_elem), _c(p.faces, np.int32).ravel(), _c(p.face_elem, np.int32),
            _c(p.traction, np.float64).ravel(), stage, C.byref(out))
        c = self._take(out)
        self.L.fo_free_csr(C.byref(out))
        return c

    def scalar_system(self, p, stage: int = 1):
        m = p.mesh
        out = _FoCsr()
        self.L.fo_scalar_system(
            m.n_nodes, _c(m.xyz, np.float64).ravel(), m.n_tets, _c(m.tets, np.int32).ravel(), _c(m.mat, np.int32),
            len(p.sigma), _c(p.sigma, np.float64), len(p.bc_nodes), _c(p.bc_nodes, np.int32),
            _c(p.bc_values, np.float64), stage, C.byref(out))
        c = self._take(out)
        self.L.fo_free_csr(C.byref(out))
        return c

    def spmv(self, A, x):
        y = np.zeros(A.n)
        self.L.fo_spmv(A.n, _c(A.row_ptr, np.int32), _c(A.col, np.int32), _c(A.val, np.float64), _c(x, np.float64), y)
        return y

    def _solve(self, fn, A, X0, *extra):
        X = _c(A.X if X0 is None else X0, np.float64).copy()
        it = C.c_int(0)
        res = fn(A.n, _c(A.row_ptr, np.int32), _c(A.col, np.int32), _c(A.val, np.float64), _c(A.F, np.float64), X,
                 *extra, C.byref(it))
        return X, res, it.value

    def cg(self, A, X0=None, maxiter=100000, tol=1e-10):
        return self._solve(self.L.fo_cg, A, X0, maxiter, tol)

    def pcg_ssor(self, A, X0=None, maxiter=100000, tol=1e-10, w=0.75):
        return self._solve(self.L.fo_pcg_ssor, A, X0, maxiter, tol, w)

    def pcg_jacobi(self, A, X0=None, maxiter=100000, tol=1e-10):
        return self._solve(self.L.fo_pcg_jacobi, A, X0, maxiter, tol)

    def minres(self, A, X0=None, maxiter=1000000, tol=1e-8):
        """Jacobi-scaled MINRES in FP64 refinement to ||F - AX|| <= tol ||F|| (not a reference routine)."""
        return self._solve(self.L.fo_minres, A, X0, maxiter, tol)

    def bicgstab(self, A, X0=None, maxiter=100000, tol=1e-10):
        return self._solve(self.L.fo_bicgstab, A, X0, maxiter, tol)

    def gmres(self, A, X0=None, m=50, maxiter=100000, tol=1e-10):
        return self._solve(self.L.fo_gmres, A, X0, m, maxiter, tol)

    def gmres_ref(self, A, X0=None, maxiter=50, tol=1e-10):
        """Modifies copies of A.val / A.F the way the reference modifies its members."""
        from . import Csr
        B = Csr(A.row_ptr, A.col, A.val.copy(), A.F.copy(), A.X.copy())
        X = _c(B.X if X0 is None else X0, np.float64).copy()
        it = C.c_int(0)
        res = self.L.fo_gmres_ref(B.n, _c(B.row_ptr, np.int32), _c(B.col, np.int32), B.val, B.F, X, maxiter, tol,
                                  C.byref(it))
        return X, res, it.value

    def driver_loop(self, A, loop, min_residual=1e-10, w=0.75, solver=None):
        """The FEM drivers' restart loop around SSOR(w)-PCG (loop 0: FEM_forBaseEliptic,
        FEM/FEM.h:627-695, which sets X = F first; loop 1: FEM_forElasticDeformation,
        FEM/FEM.h:1853-1939), from X = A.X.  Each solve gets maxiter = n (at most n - 1 iterations) and
        the needed residual 10^-(ii+1); a solve that reaches min_residual is not copied into the best
        solution (the reference breaks before the copy), and X ends as the best solution.  Returns
        (X, best_residual, [(needed, residual, iterations) per solve]).  solver(A, X, maxiter, tol)
        -> (X, residual, iterations) replaces the solve (default: this restatement's SSOR-PCG)."""
        solve = solver or (lambda B, X, maxiter, tol: self.pcg_ssor(B, X0=X, maxiter=maxiter, tol=tol, w=w))
        X = _c(A.X, np.float64).copy()
        best = X.copy()
        if loop == 0:
            X = _c(A.F, np.float64).copy()
        current, best_res = 1.0, 1e25
        max_steps, ii = (5, 0) if loop == 0 else (4, 1)
        log = []
        i = 0
        while i <= max_steps:
            needed = 10.0 ** (-1 * (ii + 1))
            if loop == 1 or current > needed:
                X, res, it = solve(A, X, A.n, needed)
                current = abs(res)
                log.append((needed, current, it))
            stop = False
            if current < needed:
                i = 0
                ii += 1
                if loop == 0 and current > best_res + 1e-10:
                    stop = True
            if not stop and current <= min_residual:
                best_res = current
                stop = True
            if stop:
                break
            if current < best_res:
                best_res = current
                best = X.copy()
            i += 1
        return best, best_res, log

    def ssor_apply(self, A, r, w=0.75):
        z = np.zeros(A.n)
        self.L.fo_ssor_apply(A.n, _c(A.row_ptr, np.int32), _c(A.col, np.int32), _c(A.val, np.float64), w,
                             _c(r, np.float64), z)
        return z


_port = None


def port() -> PortLib:
    global _port
    if _port is None:
        _port = PortLib()
    return _port


def port_available() -> bool:
    return os.path.exists(PORT_SO)
