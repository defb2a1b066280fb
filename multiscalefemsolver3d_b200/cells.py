"""Python view of the batched MsFEM cell problems (include/msfem_b200.h,
msfem_batch_* and msfem_cells_*).  Every call goes through libmsfem_b200.so.

`Cells` mirrors Grid_forMech_Poly_Order1::CreateFunctionalSpaces
(MsFEM/MsFEM_Grid.h:4795-5759) for a whole batch of macro cells: build_bases()
solves all edge, face and volume problems on the GPU and bases() returns the
8 vector basis functions of every cell, node-major [n_nodes, 8, 3].

`BatchSystems` is the batched form of the reference's cell drivers
FEM_2D/FEM_3D_forElasticDeformation (FEM/FEM.h:4367, :2970): independent
Dirichlet problems with zero source, several right-hand sides each.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import FP32_IR, FP64, check, load

__all__ = ["Cells", "BatchSystems", "FP64", "FP32_IR"]


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class BatchSystems:
    def __init__(self, dim, node_off, xyz, elem_off, elems, mat, E, nu, fixed, n_rhs):
        L = load()
        self._keep = [_c(node_off, np.int64), _c(xyz, np.float64), _c(elem_off, np.int64), _c(elems, np.int32),
                      _c(mat, np.int32), _c(E, np.float64), _c(nu, np.float64), _c(fixed, np.uint8)]
        no, xy, eo, el, mt, e, n, fx = self._keep
        self.n_sys = no.size - 1
        self.n_nodes = int(no[-1])
        self.R = n_rhs
        h = C.c_void_p()
        check(L.msfem_batch_create(dim, self.n_sys, _p(no), _p(xy), _p(eo), _p(el), _p(mt), e.size, _p(e), _p(n),
                                   _p(fx), n_rhs, 0, C.byref(h)), "batch_create")
        self.h = h

    def solve(self, x, precision=FP32_IR, tol=1e-8, maxiter=5000, threads=0):
        """x: [n_nodes, R, 3] with the Dirichlet values at fixed nodes; returns (x, rc)."""
        x = _c(x, np.float64).copy()
        rc = check(load().msfem_batch_solve(self.h, _p(x), precision, tol, maxiter, threads, 0), "batch_solve")
        return x, rc

    def report(self):
        it = np.zeros(self.n_sys, np.int32)
        out = np.zeros(self.n_sys, np.int32)
        rel = np.zeros(self.n_sys)
        ms = C.c_double()
        check(load().msfem_batch_report(self.h, _p(it), _p(out), _p(rel), C.byref(ms)), "batch_report")
        return {"inner": it, "outer": out, "rel": rel, "ms": ms.value}

    def close(self):
        if getattr(self, "h", None):
            load().msfem_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def order2_edge_order(cell_vertex):
    """[n_cells, 12]: the cell-local edge of each Order2 edge basis (host computation in the
    library; msfem_order2_edge_order)."""
    cv = _c(cell_vertex, np.int32)
    out = np.empty((cv.shape[0], 12), np.int32)
    check(load().msfem_order2_edge_order(cv.shape[0], _p(cv), _p(out)), "order2_edge_order")
    return out


class Cells:
    def __init__(self, cm):
        """cm: meshgen.CellMeshes (or any object with the same fields)."""
        L = load()
        self._keep = [_c(cm.node_off, np.int64), _c(cm.xyz, np.float64), _c(cm.tet_off, np.int64),
                      _c(cm.tets, np.int32), _c(cm.mat, np.int32), _c(cm.box, np.float64), _c(cm.E, np.float64),
                      _c(cm.nu, np.float64)]
        no, xy, to, te, mt, bx, e, n = self._keep
        self.n_cells = no.size - 1
        self.n_nodes = int(no[-1])
        h = C.c_void_p()
        check(L.msfem_cells_create(self.n_cells, _p(no), _p(xy), _p(to), _p(te), _p(mt), _p(bx), e.size, _p(e), _p(n),
                                   0, C.byref(h)), "cells_create")
        self.h = h

    def build_bases(self, precision=FP32_IR, tol=1e-8, maxiter=5000, threads=0):
        """threads = CTA size of the persistent solves; 0 autotunes it on the first build."""
        return check(load().msfem_cells_build_bases(self.h, precision, tol, maxiter, threads), "cells_build_bases")

    def set_face_material(self, mode: str):
        """"zero" (default): material 0 on the face and edge problems, as the reference's
        construction computes; "cells": face triangles and edge segments take their tetrahedra's
        material."""
        check(load().msfem_cells_set_face_material(self.h, {"cells": 0, "zero": 1}[mode]), "cells_set_face_material")

    def bases(self):
        out = np.empty((self.n_nodes, 8, 3))
        check(load().msfem_cells_get_bases(self.h, _p(out), 0), "cells_get_bases")
        return out

    def build_order2(self, cell_vertex, precision=FP32_IR, tol=1e-8, maxiter=5000, threads=0):
        """The 27 Order2 bases of every cell; cell_vertex [n_cells, 8]: the global macro vertex ids
        of each cell's corners (they fix the order of the edge bases)."""
        cv = _c(cell_vertex, np.int32)
        if cv.shape != (self.n_cells, 8):
            raise ValueError("cell_vertex must be [n_cells, 8]")
        return check(load().msfem_cells_build_order2(self.h, _p(cv), precision, tol, maxiter, threads),
                     "cells_build_order2")

    def order2_bases(self):
        out = np.empty((self.n_nodes, 27, 3))
        check(load().msfem_cells_get_order2_bases(self.h, _p(out), 0), "cells_get_order2_bases")
        return out

    def order2_macro_matrices(self):
        """[n_cells, 27, 27, 3, 3] Order2 macro element matrices of the current Order2 bases."""
        K = np.empty((self.n_cells, 27, 27, 3, 3))
        check(load().msfem_cells_order2_macro_matrices(self.h, _p(K), 0), "cells_order2_macro_matrices")
        return K

    def set_bases(self, bases):
        """Replaces every cell's bases ([n_nodes, 8, 3])."""
        b = _c(bases, np.float64)
        if b.size != 24 * self.n_nodes:
            raise ValueError("bases must be [n_nodes, 8, 3]")
        check(load().msfem_cells_set_bases(self.h, _p(b), 0), "cells_set_bases")

    def basis_residual(self):
        """Per cell ||A_II psi_I + A_IB psi_B|| / ||A_IB psi_B|| of the current bases in the cell's
        volume problems (about the solver tolerance for exact bases)."""
        rel = np.empty(self.n_cells)
        check(load().msfem_cells_basis_residual(self.h, _p(rel)), "cells_basis_residual")
        return rel

    def copy_bases_from(self, src, dst_cells):
        """Bases of cell k of `src` (a Cells) into cell dst_cells[k] of this set."""
        d = _c(dst_cells, np.int32)
        check(load().msfem_cells_copy_bases(self.h, src.h, d.size, _p(d)), "cells_copy_bases")

    def macro_matrices(self):
        """[n_cells, 8, 8, 3, 3] MsFEM macro element matrices from the current bases."""
        K = np.empty((self.n_cells, 8, 8, 3, 3))
        check(load().msfem_cells_macro_matrices(self.h, _p(K), 0), "cells_macro_matrices")
        return K

    def report(self):
        n = self.n_cells
        it, out = np.zeros(n, np.int32), np.zeros(n, np.int32)
        rel, frel, ms = np.zeros(n), np.zeros(n), np.zeros(4)
        thr = np.zeros(2, np.int32)
        check(load().msfem_cells_report(self.h, _p(it), _p(out), _p(rel), _p(frel), _p(ms), _p(thr)), "cells_report")
        return {"inner": it, "outer": out, "rel": rel, "face_rel": frel,
                "ms": dict(zip(("assemble", "edges", "faces", "volumes"), ms.tolist())),
                "threads": {"faces": int(thr[0]), "volumes": int(thr[1])}}

    def close(self):
        if getattr(self, "h", None):
            load().msfem_cells_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
