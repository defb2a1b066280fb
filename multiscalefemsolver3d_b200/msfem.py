"""The MsFEM Order1 elasticity driver on the GPU (MsFEM::MsFEM_forElasticDeformation_OrderBF1_forPoly,
MsFEM/MsFEM.h:572-1010): cell bases (Grid_forMech_Poly_Order1::CreateFunctionalSpaces), macro
element matrices (FiniteElement_forMech_Poly_Order1::SolveLocalMatrix), macro boundary loads
(BoundaryFace_forMech_Poly_Order1::SolveLocalBoundaryVector), the macro solve with Dirichlet
vertices, and the fine solution on every cell mesh.  Every step runs in libmsfem_b200.so; the
host adds the face loads into the vertex vector in item order (SummPartOfVector).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import FP32_IR, check, load
from .cells import Cells

__all__ = ["MsfemResult", "msfem_elastic_driver", "cube_macro_boundary"]


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


@dataclass
class MsfemResult:
    U: np.ndarray          # [n_vertices, 3] macro solution
    u_cells: np.ndarray    # [cell nodes, 3] fine solution on every cell mesh
    K: np.ndarray          # [n_cells, 8, 8, 3, 3] macro element matrices
    F: np.ndarray          # [n_vertices, 3] macro loads
    iterations: int
    rel_residual: float


def cube_macro_boundary(cc, traction=(0.0, 0.0, -1.0)):
    """The cube workload's macro boundary (u = 0 at z = 0, traction on z = 1) for meshgen.CubeCells:
    (Dirichlet vertices, values, load items (cell, face 5), tractions)."""
    nc = round(cc.cells.n_cells ** (1.0 / 3.0))
    V = np.arange(cc.n_coarse_vertices)
    fixed = V[V // ((nc + 1) ** 2) == 0].astype(np.int32)
    top = np.array([c for c in range(cc.cells.n_cells) if c // (nc * nc) == nc - 1], dtype=np.int32)
    items = np.stack([top, np.full(top.size, 5, np.int32)], axis=1)
    return fixed, np.zeros((fixed.size, 3)), items, np.tile(np.asarray(traction, float), (top.size, 1))


def msfem_elastic_driver(cc, fixed_vertices, fixed_values, load_items, tractions, precision=FP32_IR, tol=1e-8,
                         cell_tol=1e-10, maxiter=200000, cells: Cells | None = None) -> MsfemResult:
    """cc: meshgen.CubeCells (cells, cell_vertex, n_coarse_vertices).  Returns the macro and fine
    solutions; raises on failure."""
    L = load()
    own = cells is None
    C_ = cells if cells is not None else Cells(cc.cells)
    try:
        rc = C_.build_bases(precision=precision, tol=cell_tol)
        if rc != 0:
            raise RuntimeError(f"cell bases rc={rc}")
        # the macro phase in one device-side call: element matrices, boundary loads summed item by
        # item (SummPartOfVector), Dirichlet vertices, the macro solve and the fine reconstruction
        items = _c(load_items, np.int32).reshape(-1, 2)
        tr = _c(tractions, np.float64).reshape(-1, 3)
        cv = _c(cc.cell_vertex, np.int32)
        nv = int(cc.n_coarse_vertices)
        fv = _c(fixed_vertices, np.int32)
        fval = _c(fixed_values, np.float64).reshape(-1, 3)
        U = np.zeros((nv, 3))
        u = np.zeros((C_.n_nodes, 3))
        K = np.zeros((cv.shape[0], 8, 8, 3, 3))
        F = np.zeros((nv, 3))
        it, rel = C.c_int32(), C.c_double()
        rc = check(L.msfem_cells_order1_macro_solve(C_.h, nv, _p(cv), items.shape[0], _p(items), _p(tr), fv.size,
                                                    _p(fv), _p(fval), 0, tol, maxiter, _p(U), _p(u), _p(K), _p(F),
                                                    C.byref(it), C.byref(rel)), "cells_order1_macro_solve")
        if rc != 0:
            raise RuntimeError(f"macro solve stopped at {rel.value:.3e}")
        return MsfemResult(U=U, u_cells=u, K=K, F=F, iterations=it.value, rel_residual=rel.value)
    finally:
        if own:
            C_.close()
