"""The oracle restatement against golden vectors produced by the reference
itself (tests/golden/make_golden.py; the fixtures are committed, so these
checks need neither the reference sources nor its compiled harness)."""
import os

import numpy as np
import pytest

from multiscalefemsolver3d_b200 import meshgen

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(G, name))


def test_element_matrices(port):
    d = load("unit_tets.npz")
    for xyz, E, nu, Ke, Ks in zip(d["xyz"], d["E"], d["nu"], d["K_elastic"], d["K_scalar"]):
        np.testing.assert_allclose(port.elastic_local(xyz, E, nu), Ke, rtol=0, atol=1e-12 * np.abs(Ke).max())
        np.testing.assert_allclose(port.scalar_local(xyz, E), Ks, rtol=0, atol=1e-13 * np.abs(Ks).max())


def test_elastic_system_and_solution(port):
    d = load("elastic_n3.npz")
    p = meshgen.cube_elastic(n=int(d["n"]), jitter=float(d["jitter"]), seed=int(d["seed"]))
    assert p.mesh.xyz.sum() == pytest.approx(float(d["xyz_sum"]), rel=0, abs=1e-12)
    A = port.elastic_system(p, stage=1)
    np.testing.assert_array_equal(A.row_ptr, d["row_ptr"])
    np.testing.assert_array_equal(A.col, d["col"])
    np.testing.assert_allclose(A.val, d["val"], rtol=0, atol=1e-13 * np.abs(d["val"]).max())
    np.testing.assert_allclose(A.F, d["F"], rtol=0, atol=1e-15)
    x, res, _ = port.cg(A, tol=1e-13)
    assert np.linalg.norm(x - d["x_cg"]) / np.linalg.norm(d["x_cg"]) < 1e-11


def test_scalar_system_and_solution(port):
    d = load("scalar_n6.npz")
    p = meshgen.cube_scalar(n=int(d["n"]), n_spheres=int(d["spheres"]), rmin=float(d["rmin"]), rmax=float(d["rmax"]))
    np.testing.assert_array_equal(p.mesh.mat, d["mat"])
    A = port.scalar_system(p, stage=1)
    np.testing.assert_array_equal(A.row_ptr, d["row_ptr"])
    np.testing.assert_array_equal(A.col, d["col"])
    np.testing.assert_allclose(A.val, d["val"], rtol=0, atol=1e-13 * np.abs(d["val"]).max())
    np.testing.assert_allclose(A.F, d["F"], rtol=0, atol=1e-14)
    x, res, _ = port.cg(A, tol=1e-13)
    assert np.linalg.norm(x - d["x_cg"]) / np.linalg.norm(d["x_cg"]) < 1e-11
    # the reference driver's own output (restart loop, SSOR-PCG) agrees with its CG to ~1e-9
    assert np.linalg.norm(d["x_driver"] - d["x_cg"]) / np.linalg.norm(d["x_cg"]) < 1e-8


def test_c1_checksums(port):
    d = load("c1_elastic.npz")
    p = meshgen.cube_elastic(n=int(d["n"]), jitter=float(d["jitter"]), seed=int(d["seed"]))
    assert p.mesh.xyz.sum() == pytest.approx(float(d["xyz_sum"]), rel=0, abs=1e-9)
    A = port.elastic_system(p, stage=1)
    assert A.row_ptr[-1] == int(d["nnz"])
    assert int(A.col.astype(np.int64).sum()) == int(d["col_sum"])
    assert np.abs(A.val).sum() == pytest.approx(float(d["val_abs_sum"]), rel=1e-13)
    assert np.linalg.norm(A.val) == pytest.approx(float(d["val_fro"]), rel=1e-13)
    # the reference integrates the traction with its face quadrature applied to the base
    # tetrahedron's basis functions (alpha0 + alpha . x), which cancels ~4 digits at this
    # mesh size; the exact area/3 differs from it by up to 4e-11 relative
    np.testing.assert_allclose(A.F, d["F"], rtol=0, atol=1e-10 * np.abs(d["F"]).max())
