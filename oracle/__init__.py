"""Test infrastructure only: Python bindings of the two oracle libraries.

  ref()   -> oracle/_ref/libfemref.so      the reference's own C++ compiled from its
                                           sources (oracle/ref_harness.cpp, oracle/Makefile)
  port()  -> oracle/_build/libfemoracle.so the plain-C restatement (oracle/femoracle.c)

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm
may import this package.  The product (multiscalefemsolver3d_b200) never does.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libfemref.so")
PORT_SO = os.path.join(HERE, "_build", "libfemoracle.so")

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


class _RefCsr(C.Structure):
    _fields_ = [("n", C.c_int), ("nnz", C.c_longlong), ("row_ptr", C.POINTER(C.c_int)),
                ("col", C.POINTER(C.c_int)), ("val", C.POINTER(C.c_double)),
                ("F", C.POINTER(C.c_double)), ("X", C.POINTER(C.c_double))]


@dataclass
class Csr:
    """CSR with the diagonal included; row order [down asc, diag, up asc]."""
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


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


class RefLib:
    """The reference compiled in place (oracle/_ref/libfemref.so)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: build it with `make -C oracle ref`")
        L = C.CDLL(path)
        self.L = L
        L.ref_set_quiet.argtypes = [C.c_int]
        L.ref_free_csr.argtypes = [C.POINTER(_RefCsr)]
        L.ref_elastic_local.argtypes = [_f64p, C.c_double, C.c_double, _f64p]
        L.ref_scalar_local.argtypes = [_f64p, C.c_double, _f64p]
        mesh_args = [C.c_int, _f64p, C.c_int, _i32p, _i32p]
        L.ref_elastic_system.argtypes = mesh_args + [C.c_int, _f64p, _f64p, C.c_int, _i32p, _i32p, _f64p,
                                                     C.c_int, _i32p, _i32p, _f64p, C.c_int, C.c_int,
                                                     C.POINTER(_RefCsr), _f64p]
        L.ref_elastic_driver.argtypes = mesh_args + [C.c_int, _f64p, _f64p, C.c_int, _i32p, _i32p, _f64p,
                                                     C.c_int, _i32p, _i32p, _f64p, C.c_int, C.c_double,
                                                     _f64p, C.POINTER(C.c_double)]
        L.ref_scalar_system.argtypes = mesh_args + [C.c_int, _f64p, C.c_int, _i32p, _f64p, C.c_int, C.c_int,
                                                    C.POINTER(_RefCsr), _f64p]
        L.ref_scalar_driver.argtypes = mesh_args + [C.c_int, _f64p, C.c_int, _i32p, _f64p, C.c_int, C.c_double,
                                                    _f64p, C.POINTER(C.c_double)]
        L.ref_cssd_solve.argtypes = [C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, _f64p, C.c_int, C.c_double,
                                     C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.ref_ssor_apply.argtypes = [C.c_int, _i32p, _i32p, _f64p, C.c_double, _f64p, _f64p]
        L.ref_cell_problem.argtypes = [C.c_int, C.c_int, _f64p, C.c_int, _i32p, _i32p, C.c_int, _f64p, _f64p,
                                       C.c_int, _i32p, _f64p, C.c_double, _f64p]
        L.ref_poly_quadrature.argtypes = [_f64p, _i32p, _f64p, _f64p]
        L.ref_mech_D.argtypes = [C.c_double, C.c_double, _f64p]
        L.ref_polygon_quadrature.argtypes = [_f64p, _f64p, _f64p]
        _i = C.c_int
        _ip = C.POINTER(C.c_int)
        L.ref_read_nvtr.argtypes = [C.c_char_p, _i, _i, _i, _i, _ip, _ip, _ip, _f64p, _i32p, _i32p, _i32p, _ip]
        L.ref_read_salome.argtypes = [C.c_char_p, _i, _i, _i, _i, _ip, _ip, _f64p, _i32p, _i32p]
        L.ref_postprocess.argtypes = [_i, _f64p, _i, _i32p, _i32p, _i, _f64p, _f64p, _f64p, _f64p]
        L.ref_scalar3_local.argtypes = [_f64p, C.c_double, C.c_double, C.c_double, _f64p, _f64p]
        L.ref_scalar3_driver.argtypes = [_i, _f64p, _i, _i32p, _f64p, _f64p, _f64p, _i, _i32p, _f64p, C.c_double,
                                         _f64p]
        for f in ("ref_elastic_local", "ref_scalar_local", "ref_elastic_system", "ref_elastic_driver",
                  "ref_scalar_system", "ref_scalar_driver", "ref_cssd_solve", "ref_ssor_apply", "ref_cell_problem",
                  "ref_poly_quadrature", "ref_mech_D", "ref_polygon_quadrature", "ref_read_nvtr", "ref_read_salome", "ref_postprocess",
                  "ref_scalar3_local", "ref_scalar3_driver"):
            getattr(L, f).restype = C.c_int
        L.ref_set_quiet(1)

    @staticmethod
    def _take(out: _RefCsr) -> Csr:
        n, nnz = out.n, out.nnz
        c = Csr(
            row_ptr=np.ctypeslib.as_array(out.row_ptr, shape=(n + 1,)).copy(),
            col=np.ctypeslib.as_array(out.col, shape=(nnz,)).copy(),
            val=np.ctypeslib.as_array(out.val, shape=(nnz,)).copy(),
            F=np.ctypeslib.as_array(out.F, shape=(n,)).copy(),
            X=np.ctypeslib.as_array(out.X, shape=(n,)).copy(),
        )
        return c

    def elastic_local(self, xyz4, E=1.0, nu=0.3) -> np.ndarray:
        K = np.zeros(144)
        rc = self.L.ref_elastic_local(_c(xyz4, np.float64).ravel(), E, nu, K)
        assert rc == 0
        return K.reshape(4, 4, 3, 3)

    def scalar_local(self, xyz4, sigma=1.0) -> np.ndarray:
        K = np.zeros(16)
        rc = self.L.ref_scalar_local(_c(xyz4, np.float64).ravel(), sigma, K)
        assert rc == 0
        return K.reshape(4, 4)

    def scalar3_local(self, xyz4, S, M, f):
        """(K + M [4, 4], F [4]) of FiniteElement_forScal::SolveLocalMatrix (FEM_Grid.h:25-102)."""
        K, F = np.zeros(16), np.zeros(4)
        rc = self.L.ref_scalar3_local(_c(xyz4, np.float64).ravel(), S, M, f, K, F)
        assert rc == 0
        return K.reshape(4, 4), F

    def scalar3_driver(self, xyz, tets, S, M, f, bc_nodes, bc_values, min_residual=1e-12):
        """The three-coefficient FEM_forBaseEliptic (FEM.h:206-397) with per-element coefficients."""
        xyz = _c(xyz, np.float64)
        tets = _c(tets, np.int32)
        sol = np.zeros(xyz.shape[0])
        rc = self.L.ref_scalar3_driver(xyz.shape[0], xyz.ravel(), tets.shape[0], tets.ravel(), _c(S, np.float64),
                                       _c(M, np.float64), _c(f, np.float64), len(bc_nodes), _c(bc_nodes, np.int32),
                                       _c(bc_values, np.float64), min_residual, sol)
        assert rc == 0, rc
        return sol

    def elastic_system(self, p, stage: int = 1, nthreads: int = 1):
        m = p.mesh
        out = _RefCsr()
        t = np.zeros(2)
        rc = self.L.ref_elastic_system(
            m.n_nodes, _c(m.xyz, np.float64).ravel(), m.n_tets, _c(m.tets, np.int32).ravel(), _c(m.mat, np.int32),
            len(p.E), _c(p.E, np.float64), _c(p.nu, np.float64),
            len(p.bc_nodes), _c(p.bc_nodes, np.int32), _c(p.bc_mask, np.int32), _c(p.bc_values, np.float64).ravel(),
            len(p.face_elem), _c(p.faces, np.int32).ravel(), _c(p.face_elem, np.int32),
            _c(p.traction, np.float64).ravel(), nthreads, stage, C.byref(out), t)
        assert rc == 0, rc
        c = self._take(out)
        self.L.ref_free_csr(C.byref(out))
        return c, t

    def elastic_driver(self, p, min_residual: float = 1e-10, nthreads: int = 1):
        m = p.mesh
        sol = np.zeros(3 * m.n_nodes)
        wall = C.c_double(0)
        rc = self.L.ref_elastic_driver(
            m.n_nodes, _c(m.xyz, np.float64).ravel(), m.n_tets, _c(m.tets, np.int32).ravel(), _c(m.mat, np.int32),
            len(p.E), _c(p.E, np.float64), _c(p.nu, np.float64),
            len(p.bc_nodes), _c(p.bc_nodes, np.int32), _c(p.bc_mask, np.int32), _c(p.bc_values, np.float64).ravel(),
            len(p.face_elem), _c(p.faces, np.int32).ravel(), _c(p.face_elem, np.int32),
            _c(p.traction, np.float64).ravel(), nthreads, min_residual, sol, C.byref(wall))
        assert rc == 0, rc
        return sol, wall.value

    def scalar_system(self, p, stage: int = 1, nthreads: int = 1):
        m = p.mesh
        out = _RefCsr()
        t = np.zeros(2)
        rc = self.L.ref_scalar_system(
            m.n_nodes, _c(m.xyz, np.float64).ravel(), m.n_tets, _c(m.tets, np.int32).ravel(), _c(m.mat, np.int32),
            len(p.sigma), _c(p.sigma, np.float64), len(p.bc_nodes), _c(p.bc_nodes, np.int32),
            _c(p.bc_values, np.float64), nthreads, stage, C.byref(out), t)
        assert rc == 0, rc
        c = self._take(out)
        self.L.ref_free_csr(C.byref(out))
        return c, t

    def scalar_driver(self, p, min_residual: float = 1e-10, nthreads: int = 1):
        m = p.mesh
        sol = np.zeros(m.n_nodes)
        wall = C.c_double(0)
        rc = self.L.ref_scalar_driver(
            m.n_nodes, _c(m.xyz, np.float64).ravel(), m.n_tets, _c(m.tets, np.int32).ravel(), _c(m.mat, np.int32),
            len(p.sigma), _c(p.sigma, np.float64), len(p.bc_nodes), _c(p.bc_nodes, np.int32),
            _c(p.bc_values, np.float64), nthreads, min_residual, sol, C.byref(wall))
        assert rc == 0, rc
        return sol, wall.value

    def cssd_solve(self, method: int, A: Csr, X0=None, maxiter: int = 100000, tol: float = 1e-10, nthreads: int = 1):
        """method: 0 MSG (CG), 1 SSOR(0.75)-PCG, 2 BiCG_Stab, 3 BCG_Stab2, 4 GMRES(5)."""
        X = _c(A.X if X0 is None else X0, np.float64).copy()
        res = C.c_double(0)
        wall = C.c_double(0)
        rc = self.L.ref_cssd_solve(method, A.n, _c(A.row_ptr, np.int32), _c(A.col, np.int32), _c(A.val, np.float64),
                                   _c(A.F, np.float64), X, maxiter, tol, nthreads, C.byref(res), C.byref(wall))
        assert rc == 0, rc
        return X, res.value, wall.value

    def cell_problem(self, dim: int, xyz, elems, mat, E, nu, bc_nodes, bc_values, min_residual: float = 5e-15):
        """One MsFEM cell sub-problem (dim 1 edge, 2 face, 3 volume) through the reference's
        FEM_1D/2D/3D_forElasticDeformation; returns the solution [n_nodes, 3]."""
        xyz = _c(xyz, np.float64)
        elems = _c(elems, np.int32)
        n = xyz.shape[0]
        sol = np.zeros(3 * n)
        rc = self.L.ref_cell_problem(dim, n, xyz.ravel(), elems.shape[0], elems.ravel(), _c(mat, np.int32),
                                     len(E), _c(E, np.float64), _c(nu, np.float64), len(bc_nodes),
                                     _c(bc_nodes, np.int32), _c(bc_values, np.float64).ravel(), min_residual, sol)
        assert rc == 0, rc
        return sol.reshape(n, 3)

    def poly_quadrature(self, xyz8, faces):
        """The reference's macro-element quadrature: (points [96, 3], weights [96])."""
        pts, w = np.zeros(288), np.zeros(96)
        rc = self.L.ref_poly_quadrature(_c(xyz8, np.float64).ravel(), _c(faces, np.int32).ravel(), pts, w)
        assert rc == 0, rc
        return pts.reshape(96, 3), w

    def polygon_quadrature(self, xyz4):
        """The reference's macro-face quadrature: (points [16, 3], weights [16])."""
        pts, w = np.zeros(48), np.zeros(16)
        assert self.L.ref_polygon_quadrature(_c(xyz4, np.float64).ravel(), pts, w) == 0
        return pts.reshape(16, 3), w

    def read_nvtr(self, directory, k, cap_v, cap_e, cap_idx):
        """The reference's ReadFromNVTR: (xyz [nv, 3], elements (list of index arrays), nvkat,
        read_from_zero)."""
        nv, ne, ni, rz = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        xyz, idx = np.zeros(3 * cap_v), np.zeros(cap_idx, np.int32)
        ln, kat = np.zeros(cap_e, np.int32), np.zeros(cap_e, np.int32)
        rc = self.L.ref_read_nvtr(str(directory).encode(), k, cap_v, cap_e, cap_idx, C.byref(nv), C.byref(ne), C.byref(ni),
                                  xyz, idx, ln, kat, C.byref(rz))
        assert rc == 0, rc
        assert nv.value <= cap_v and ne.value <= cap_e and ni.value <= cap_idx
        off = np.concatenate([[0], np.cumsum(ln[:ne.value])])
        elems = [idx[off[e]:off[e + 1]].copy() for e in range(ne.value)]
        return xyz[:3 * nv.value].reshape(-1, 3), elems, kat[:ne.value].copy(), bool(rz.value)

    def read_salome(self, path, dim, map_size, cap_v, cap_e):
        """The reference's ReadFromSalomeDat: (xyz, elements [ne, dim + 1], vertex_map or None)."""
        nv, ne = C.c_int(), C.c_int()
        xyz, el = np.zeros(3 * cap_v), np.zeros((dim + 1) * cap_e, np.int32)
        vm = np.zeros(cap_v, np.int32)
        rc = self.L.ref_read_salome(str(path).encode(), dim, map_size, cap_v, cap_e, C.byref(nv), C.byref(ne), xyz, el, vm)
        assert rc == 0, rc
        return (xyz[:3 * nv.value].reshape(-1, 3), el[:(dim + 1) * ne.value].reshape(-1, dim + 1),
                vm[:nv.value].copy() if map_size >= 0 else None)

    def postprocess(self, mesh, E, nu, solution):
        """[n_tets, 19] per element at its centroid: U, dU (row a = grad u_a), sigma (xx yy zz yz xz
        xy) with the element's material, von Mises (FEM/FEM_Grid.h:3289-3365)."""
        out = np.zeros(19 * mesh.n_tets)
        E = _c(E, np.float64)
        rc = self.L.ref_postprocess(mesh.n_nodes, _c(mesh.xyz, np.float64).ravel(), mesh.n_tets,
                                    _c(mesh.tets, np.int32).ravel(), _c(mesh.mat, np.int32), E.size, E,
                                    _c(nu, np.float64), _c(solution, np.float64).ravel(), out)
        assert rc == 0, rc
        return out.reshape(-1, 19)

    def mech_D(self, E, nu):
        D = np.zeros(36)
        assert self.L.ref_mech_D(E, nu, D) == 0
        return D.reshape(6, 6)

    def ssor_apply(self, A: Csr, r, w: float = 0.75):
        z = np.zeros(A.n)
        rc = self.L.ref_ssor_apply(A.n, _c(A.row_ptr, np.int32), _c(A.col, np.int32), _c(A.val, np.float64), w,
                                   _c(r, np.float64), z)
        assert rc == 0
        return z


_ref_singleton = None


def ref() -> RefLib:
    global _ref_singleton
    if _ref_singleton is None:
        _ref_singleton = RefLib()
    return _ref_singleton


def ref_available() -> bool:
    return os.path.exists(REF_SO)


from .port import PortLib, port, port_available  # noqa: E402  (restatement bindings)
