"""The C-ABI library loads and exports every entry point include/msfem_b200.h
declares (no compute call: this runs on machines without a GPU)."""
import ctypes
import os
import re
import subprocess

from multiscalefemsolver3d_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not h.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(msfem_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_boundary():
    names = declared_functions()
    for required in ("msfem_system_create", "msfem_assemble_scalar", "msfem_assemble_elastic", "msfem_add_traction",
                     "msfem_apply_dirichlet", "msfem_solve", "msfem_export_csr", "msfem_fem_scalar_driver",
                     "msfem_fem_elastic_driver"):
        assert required in names


def test_library_exports_every_declared_symbol(lib):
    for name in declared_functions():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (msfem_\w+)", out))
    assert set(declared_functions()) <= exported


def test_binding_covers_the_header(lib):
    assert set(_lib.EXPORTED) == set(declared_functions())


def test_version_and_error_string(lib):
    assert lib.msfem_version() >= 100
    assert isinstance(lib.msfem_last_error(), bytes)


def test_null_handle_is_an_error_not_a_crash(lib):
    # argument checks run before any CUDA call
    assert lib.msfem_system_info(None, None, None, None) == -1
    assert lib.msfem_system_destroy(None) == 0
    out = ctypes.c_void_p()
    assert lib.msfem_system_create(5, 10, None, 10, None, None, 0, ctypes.byref(out)) == -1


def test_new_entry_points_refuse_null_handles(lib):
    """The device-side Order2 macro calls and the scaled matrix-free product check their handles
    before any CUDA call: a null handle is an argument error with a message, not a crash."""
    out = ctypes.c_void_p()
    assert lib.msfem_cells_order2_macro_system(None, 10, None, ctypes.byref(out)) == -1
    assert b"msfem_cells_order2_macro_system" in lib.msfem_last_error()
    assert lib.msfem_cells_order2_dirichlet(None, 10, None, 1, None, 0, None, 1, None, None, None, None,
                                            None) == -1
    assert b"msfem_cells_order2_dirichlet" in lib.msfem_last_error()
    it, rel = ctypes.c_int32(), ctypes.c_double()
    assert lib.msfem_cells_order2_macro_solve(None, 10, None, 1, None, 0, None, 0, None, None, None, None, 0,
                                              None, None, 0, 1e-8, 10, None, ctypes.byref(it),
                                              ctypes.byref(rel)) == -1
    assert b"msfem_cells_order2_macro_solve" in lib.msfem_last_error()
    assert lib.msfem_kuhn_spmv_scaled32(None, None, None, 0) == -1
