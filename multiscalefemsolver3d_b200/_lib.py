"""ctypes binding of libmsfem_b200.so (the C ABI in include/msfem_b200.h).

The library is loaded from the package directory; if it is missing the import
fails loudly (there is no fallback path).  Build it with
`python -m multiscalefemsolver3d_b200.build`.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libmsfem_b200.so")

MSFEM_OK = 0
MSFEM_NOT_CONVERGED = 1
MSFEM_ERR_ARGUMENT = -1
MSFEM_ERR_LIMIT = -4

SCALAR, ELASTIC = 0, 1
CG, PCG_JACOBI, BICGSTAB, GMRES, MINRES, PCG_SSOR = 0, 1, 2, 3, 4, 5
LOOP_SCALAR, LOOP_ELASTIC = 0, 1
FP64, FP32_IR, FP64_REFERENCE = 0, 1, 2
ROW_ONLY, ROW_AND_COLUMN = 0, 1


class Stats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int),
        ("outer_iterations", C.c_int),
        ("rel_residual", C.c_double),
        ("ms_portrait", C.c_double),
        ("ms_assemble", C.c_double),
        ("ms_dirichlet", C.c_double),
        ("ms_solve", C.c_double),
        ("ms_spmv", C.c_double),
        ("n_colors", C.c_int),
        ("kernel_launches", C.c_int),
        ("total_launches", C.c_int64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# (name, restype, argtypes); arrays are passed as void pointers so that numpy
# host arrays and CUDA device pointers (torch .data_ptr()) both fit
_P = C.c_void_p
_SIGS = [
    ("msfem_last_error", C.c_char_p, []),
    ("msfem_version", C.c_int, []),
    ("msfem_system_create", C.c_int, [C.c_int, C.c_int, _P, C.c_int, _P, _P, C.c_int, C.POINTER(C.c_void_p)]),
    ("msfem_system_from_cssd", C.c_int, [C.c_int, _P, _P, _P, _P, _P, _P, _P, _P, _P, C.POINTER(C.c_void_p)]),
    ("msfem_xfem_system", C.c_int, [C.c_int, _P, C.c_int, _P, _P, C.c_int, _P, _P, _P, _P, C.c_int,
                                    C.POINTER(C.c_void_p)]),
    ("msfem_system_destroy", C.c_int, [C.c_void_p]),
    ("msfem_system_info", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int64), C.POINTER(C.c_int)]),
    ("msfem_get_stats", C.c_int, [C.c_void_p, C.POINTER(Stats)]),
    ("msfem_get_stream", C.c_void_p, [C.c_void_p]),
    ("msfem_clear", C.c_int, [C.c_void_p]),
    ("msfem_assemble_scalar", C.c_int, [C.c_void_p, _P, C.c_int]),
    ("msfem_assemble_scalar3", C.c_int, [C.c_void_p, _P, _P, _P, C.c_int]),
    ("msfem_assemble_elastic", C.c_int, [C.c_void_p, _P, _P, C.c_int]),
    ("msfem_assemble_elastic_textbook", C.c_int, [C.c_void_p, _P, _P, C.c_int]),
    ("msfem_add_traction", C.c_int, [C.c_void_p, C.c_int, _P, _P, C.c_int]),
    ("msfem_add_rhs", C.c_int, [C.c_void_p, _P, C.c_int]),
    ("msfem_apply_dirichlet", C.c_int, [C.c_void_p, C.c_int, _P, _P, C.c_int, C.c_int]),
    ("msfem_set_x", C.c_int, [C.c_void_p, _P, C.c_int]),
    ("msfem_get_x", C.c_int, [C.c_void_p, _P, C.c_int]),
    ("msfem_get_f", C.c_int, [C.c_void_p, _P, C.c_int]),
    ("msfem_copy_f_to_x", C.c_int, [C.c_void_p]),
    ("msfem_solve", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                              C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    ("msfem_set_ssor_omega", C.c_int, [C.c_void_p, C.c_double]),
    ("msfem_ssor_apply", C.c_int, [C.c_void_p, _P, _P, C.c_int]),
    ("msfem_solve_driver_loop", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double,
                                          C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("msfem_spmv", C.c_int, [C.c_void_p, _P, _P, C.c_int]),
    ("msfem_spmv_scaled32", C.c_int, [C.c_void_p, _P, _P, C.c_int]),
    ("msfem_set_kuhn_grid", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int]),
    ("msfem_release_cached_memory", None, []),
    ("msfem_kuhn_spmv", C.c_int, [C.c_void_p, _P, _P, C.c_int]),
    ("msfem_kuhn_spmv_scaled32", C.c_int, [C.c_void_p, _P, _P, C.c_int]),
    ("msfem_export_csr", C.c_int, [C.c_void_p, _P, _P, _P, C.c_int]),
    ("msfem_bench_spmv", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    ("msfem_residual_noalloc", C.c_int, [C.c_int, _P, _P, _P, _P, _P, _P, _P, C.c_void_p]),
    ("msfem_fem_scalar_driver", C.c_int, [C.c_int, _P, C.c_int, _P, _P, C.c_int, _P, C.c_int, _P, _P, C.c_int,
                                          C.c_int, C.c_double, C.c_int, _P, C.POINTER(Stats)]),
    ("msfem_fem_elastic_driver", C.c_int, [C.c_int, _P, C.c_int, _P, _P, C.c_int, _P, _P, C.c_int, _P, _P, _P,
                                           C.c_int, _P, _P, C.c_int, C.c_int, C.c_double, C.c_int, _P,
                                           C.POINTER(Stats)]),
    ("msfem_batch_create", C.c_int, [C.c_int, C.c_int, _P, _P, _P, _P, _P, C.c_int, _P, _P, _P, C.c_int, C.c_int,
                                     C.POINTER(C.c_void_p)]),
    ("msfem_batch_solve", C.c_int, [C.c_void_p, _P, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int]),
    ("msfem_batch_report", C.c_int, [C.c_void_p, _P, _P, _P, C.POINTER(C.c_double)]),
    ("msfem_batch_destroy", None, [C.c_void_p]),
    ("msfem_cells_create", C.c_int, [C.c_int, _P, _P, _P, _P, _P, _P, C.c_int, _P, _P, C.c_int,
                                     C.POINTER(C.c_void_p)]),
    ("msfem_cells_build_bases", C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_int]),
    ("msfem_cells_get_bases", C.c_int, [C.c_void_p, _P, C.c_int]),
    ("msfem_cells_set_face_material", C.c_int, [C.c_void_p, C.c_int]),
    ("msfem_cells_build_order2", C.c_int, [C.c_void_p, _P, C.c_int, C.c_double, C.c_int, C.c_int]),
    ("msfem_order2_edge_order", C.c_int, [C.c_int, _P, _P]),
    ("msfem_cells_get_order2_bases", C.c_int, [C.c_void_p, _P, C.c_int]),
    ("msfem_cells_order2_macro_matrices", C.c_int, [C.c_void_p, _P, C.c_int]),
    ("msfem_cells_order2_macro_system", C.c_int, [C.c_void_p, C.c_int, _P, C.POINTER(C.c_void_p)]),
    ("msfem_cells_order2_dirichlet", C.c_int, [C.c_void_p, C.c_int, _P, C.c_int, _P, C.c_int, _P, C.c_int, _P, _P, _P,
                                               _P, _P]),
    ("msfem_cells_order2_macro_solve", C.c_int, [C.c_void_p, C.c_int, _P, C.c_int, _P, C.c_int, _P, C.c_int, _P, _P,
                                                 _P, _P, C.c_int, _P, _P, C.c_int, C.c_double, C.c_int, _P,
                                                 C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    ("msfem_cells_report", C.c_int, [C.c_void_p, _P, _P, _P, _P, _P, _P]),
    ("msfem_cells_macro_matrices", C.c_int, [C.c_void_p, _P, C.c_int]),
    ("msfem_cells_face_loads", C.c_int, [C.c_void_p, C.c_int, _P, _P, _P]),
    ("msfem_cells_reconstruct", C.c_int, [C.c_void_p, C.c_int, _P, _P, _P]),
    ("msfem_cells_order1_macro_solve", C.c_int, [C.c_void_p, C.c_int, _P, C.c_int, _P, _P, C.c_int, _P, _P, C.c_int,
                                                  C.c_double, C.c_int, _P, _P, _P, _P, C.POINTER(C.c_int32),
                                                  C.POINTER(C.c_double)]),
    ("msfem_postprocess_elastic", C.c_int, [C.c_void_p, C.c_int, _P, _P, _P, C.c_int]),
    ("msfem_cells_set_bases", C.c_int, [C.c_void_p, _P, C.c_int]),
    ("msfem_cells_basis_residual", C.c_int, [C.c_void_p, _P]),
    ("msfem_cells_copy_bases", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, _P]),
    ("msfem_cells_destroy", None, [C.c_void_p]),
    ("msfem_macro_solve", C.c_int, [C.c_int, C.c_int, _P, _P, _P, C.c_int, _P, _P, C.c_int, C.c_double, C.c_int,
                                    _P, _P, _P]),
    ("msfem_coarse_create", C.c_int, [C.c_void_p, C.c_void_p, _P, C.c_int, _P, _P, C.c_int, _P,
                                      C.POINTER(C.c_void_p)]),
    ("msfem_coarse_info", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    ("msfem_coarse_matrix", C.c_int, [C.c_void_p, _P, _P]),
    ("msfem_coarse_apply", C.c_int, [C.c_void_p, _P, _P]),
    ("msfem_solve_twolevel", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_double, C.POINTER(C.c_double),
                                       C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    ("msfem_coarse_bench_smoother", C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int64)]),
    ("msfem_coarse_set_smoother", C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_int]),
    ("msfem_coarse_set_matrix_free", C.c_int, [C.c_void_p, C.c_int]),
    ("msfem_coarse_stats", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_int)]),
    ("msfem_coarse_destroy", None, [C.c_void_p]),
    ("msfem_net_param_count", C.c_int, []),
    ("msfem_net_create", C.c_int, [C.c_uint64, C.c_double, C.c_double, C.POINTER(C.c_void_p)]),
    ("msfem_net_get_params", C.c_int, [C.c_void_p, _P]),
    ("msfem_net_set_params", C.c_int, [C.c_void_p, _P]),
    ("msfem_net_voxelise", C.c_int, [C.c_void_p, C.c_void_p, _P]),
    ("msfem_net_add_cells", C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]),
    ("msfem_net_train", C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_uint64, _P]),
    ("msfem_net_loss_grad", C.c_int, [C.c_void_p, C.c_int, _P, _P, _P, _P]),
    ("msfem_net_forward", C.c_int, [C.c_void_p, C.c_int, _P, _P]),
    ("msfem_net_predict", C.c_int, [C.c_void_p, C.c_void_p, _P]),
    ("msfem_net_set_tensor_path", C.c_int, [C.c_void_p, C.c_int]),
    ("msfem_net_destroy", C.c_int, [C.c_void_p]),
]

EXPORTED = [name for name, _, _ in _SIGS]

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Loads the library (once).  Raises if it is missing: no CPU fallback exists."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing; build it with `python -m multiscalefemsolver3d_b200.build`")
    L = C.CDLL(path)
    for name, res, args in _SIGS:
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


class MsfemError(RuntimeError):
    def __init__(self, rc: int, where: str):
        msg = load().msfem_last_error().decode(errors="replace")
        super().__init__(f"{where} failed ({rc}): {msg}")
        self.rc = rc


def check(rc: int, where: str) -> int:
    if rc < 0:
        raise MsfemError(rc, where)
    return rc
