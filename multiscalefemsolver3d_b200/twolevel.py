"""Two-level preconditioner with the MsFEM coarse space (include/msfem_b200.h,
msfem_coarse_* and msfem_solve_twolevel): a fine elasticity System, the macro
cells covering its mesh with their Order1 bases (cells.Cells), and the solve
that uses them.  Every call goes through libmsfem_b200.so.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import FP32_IR, FP64, check, load

__all__ = ["TwoLevel", "FP64", "FP32_IR"]


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class TwoLevel:
    def __init__(self, system, cells, cube_cells, fixed_dofs):
        """system: fem.System (elasticity, assembled, Dirichlet applied); cells: cells.Cells with
        bases built; cube_cells: meshgen.CubeCells (maps); fixed_dofs: the fine Dirichlet DOFs."""
        L = load()
        self._keep = [_c(cube_cells.cell_node_global, np.int32), _c(cube_cells.cell_vertex, np.int32),
                      _c(cube_cells.cell_color, np.int32), _c(fixed_dofs, np.int32)]
        cng, cv, col, fx = self._keep
        self.system = system
        self.cells = cells
        self.n_cells = cv.shape[0]
        h = C.c_void_p()
        check(L.msfem_coarse_create(system.h, cells.h, _p(cng), int(cube_cells.n_coarse_vertices), _p(cv), _p(col),
                                    fx.size, _p(fx), C.byref(h)), "coarse_create")
        self.h = h
        n, ms = C.c_int(), C.c_double()
        check(L.msfem_coarse_info(h, C.byref(n), C.byref(ms)), "coarse_info")
        self.n_coarse_dofs, self.ms_setup = n.value, ms.value

    def solve(self, tol=1e-8, maxiter=200000, precision=FP32_IR):
        rel, it, out = C.c_double(), C.c_int(), C.c_int()
        rc = check(load().msfem_solve_twolevel(self.system.h, self.h, precision, maxiter, tol, C.byref(rel),
                                               C.byref(it), C.byref(out)), "solve_twolevel")
        return rel.value, it.value, out.value, rc

    def set_smoother(self, textbook_system, degree=5, ratio=100.0, half_matrix=False, matrix_free=False):
        """Multiplicative cycle with Chebyshev smoothing on the textbook-orientation system
        (fem.System assembled with assemble_elastic_textbook, same Dirichlet rows); half_matrix
        stores the smoother's matrix values in FP16; matrix_free applies the operator from the
        tetrahedra's materials on the system's Kuhn grid (System.set_kuhn_grid).  ratio > 1: the
        first-kind Chebyshev polynomial for [lambda_max / ratio, lambda_max]; ratio 0: the
        fourth-kind polynomial on [0, lambda_max].  The default degree and spectrum ratio were the
        fastest of a sweep on the 128^3 elasticity case."""
        self._text = textbook_system
        storage = 2 if matrix_free else (1 if half_matrix else 0)
        check(load().msfem_coarse_set_smoother(self.h, textbook_system.h, degree, ratio, storage),
              "coarse_set_smoother")

    def set_matrix_free(self, on=True):
        """MINRES's FP64 products with the fine matrix formed matrix-free on its Kuhn grid."""
        check(load().msfem_coarse_set_matrix_free(self.h, int(bool(on))), "coarse_set_matrix_free")

    def bench_smoother(self, reps=100):
        """(ms per Chebyshev step, algorithmic bytes per step) of the cycle's smoothing kernel."""
        ms, nb = C.c_double(), C.c_int64()
        check(load().msfem_coarse_bench_smoother(self.h, reps, C.byref(ms), C.byref(nb)), "coarse_bench_smoother")
        return ms.value, nb.value

    def stats(self):
        """{'trilinear_cells', 'lambda_max', 'widened'}: see msfem_coarse_stats."""
        t, w = C.c_int(), C.c_int()
        lm = C.c_double()
        check(load().msfem_coarse_stats(self.h, C.byref(t), C.byref(lm), C.byref(w)), "coarse_stats")
        return {"trilinear_cells": t.value, "lambda_max": lm.value, "widened": w.value}

    def coarse_matrix(self):
        A = np.empty((self.n_coarse_dofs, self.n_coarse_dofs))
        cdof = np.empty((self.n_cells, 8, 3), np.int32)
        check(load().msfem_coarse_matrix(self.h, _p(A), _p(cdof)), "coarse_matrix")
        return A, cdof

    def apply(self, r):
        r = _c(r, np.float32)
        y = np.empty_like(r)
        check(load().msfem_coarse_apply(self.h, _p(r), _p(y)), "coarse_apply")
        return y

    def close(self):
        if getattr(self, "h", None):
            load().msfem_coarse_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
