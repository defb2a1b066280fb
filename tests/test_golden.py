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


def _msfem_groups(vxyz):
    bot = np.nonzero(np.abs(vxyz[:, 2]) < 1e-12)[0]
    top = np.nonzero(np.abs(vxyz[:, 2] - 1) < 1e-12)[0]
    return [(bot, (0.0, 0.0, 0.0), (1, 1, 1)), (top, (0.01, -0.02, 0.05), (1, 1, 1))]


def test_msfem_order1_against_reference_run():
    """Order1 bases (material 0 on faces and edges, as the reference) and the Order1 driver's macro
    solution against the reference's whole Order1 run."""
    import types

    from oracle import cells as oc
    from oracle import msfem as om
    from oracle import order2 as o2
    d = load("msfem_order1.npz")
    vxyz, cv, cm = o2.graded_cells(2, 4, 0.5)
    assert abs(cm.xyz.sum() - float(d["xyz_sum"])) < 1e-9
    bases = [oc.order1_bases(*cm.cell(c)[:3], cm.cell(c)[3], cm.E, cm.nu, face_material="zero")
             for c in range(cm.n_cells)]
    for c in (0, 7):
        np.testing.assert_allclose(bases[c], d[f"bases_{c}"], rtol=0, atol=1e-11)
    groups = _msfem_groups(vxyz)
    cc = types.SimpleNamespace(cells=cm, cell_vertex=cv, n_coarse_vertices=vxyz.shape[0])
    fv = np.concatenate([g[0] for g in groups])
    vals = np.concatenate([np.tile(g[1], (len(g[0]), 1)) for g in groups])
    U, _, _, _ = om.driver(cc, np.concatenate(bases), fv, vals, [], [], cm.E[0], cm.nu[0])
    assert np.linalg.norm(U - d["solution"]) <= 1e-9 * np.linalg.norm(d["solution"])


def test_msfem_order2_against_reference_run():
    """Order2 bases, macro element matrix, DOF numbering and the whole Order2 driver's macro
    solution against the reference's own run."""
    from oracle import order2 as o2
    d = load("msfem_order2.npz")
    vxyz1, cv1, cm1 = o2.graded_cells(1, 4, 0.5)
    assert abs(cm1.xyz.sum() - float(d["xyz_sum_1"])) < 1e-9
    xyz, tets, mat, box = cm1.cell(0)
    B = o2.order2_bases(xyz, tets, mat, box, cm1.E, cm1.nu, cv1[0])
    np.testing.assert_allclose(B, d["bases"], rtol=0, atol=1e-11 * np.abs(d["bases"]).max())
    K = o2.macro_element_matrix(xyz, tets, B, box, cm1.E[0], cm1.nu[0]).transpose(0, 2, 1, 3).reshape(81, 81)
    np.testing.assert_allclose(K, d["K"], rtol=0, atol=1e-11 * np.abs(d["K"]).max())
    vxyz, cv, cm = o2.graded_cells(2, 4, 0.5)
    assert abs(cm.xyz.sum() - float(d["xyz_sum_2"])) < 1e-9
    np.testing.assert_array_equal(o2.macro_topology(cv)[3], d["cell_dofs"])
    x = o2.order2_driver(vxyz, cv, cm, _msfem_groups(vxyz))
    assert np.linalg.norm(x - d["solution"]) <= 1e-9 * np.linalg.norm(d["solution"])
