"""Batched MsFEM cell problems on the GPU vs the oracle (oracle/cells.py, pinned
against the reference's FEM_1D/2D/3D cell drivers in test_cells_oracle.py).

Bars: each batched Dirichlet problem within 1e-8 relative (max norm over the
solution) of the exact sparse-LU solution; Order1 bases within 1e-8 of the
oracle's chain; at the full cell sizes ({8,12,16,20}^3 hexes) the size-
independent properties: the 8 bases of a cell add up to (1,1,1) at every node,
basis v is (1,1,1) at vertex v and 0 at the other vertices, and two builds give
the same bits.
"""
import numpy as np
import pytest

from multiscalefemsolver3d_b200 import _lib, meshgen
from multiscalefemsolver3d_b200.cells import FP32_IR, FP64, BatchSystems, Cells
from oracle import cells as ocells

pytestmark = pytest.mark.gpu

SOL_TOL = 1e-8


def _volume_batch(n_sys=5, R=8, seed=0):
    rng = np.random.default_rng(seed)
    node_off, elem_off, xyzs, elems, mats, fixeds, sizes = [0], [0], [], [], [], [], []
    for s in range(n_sys):
        m = meshgen.kuhn_cube(3 + s % 3, jitter=0.15, seed=seed + s)
        bnd = np.any((m.xyz < 1e-12) | (m.xyz > 1 - 1e-12), axis=1)
        xyzs.append(m.xyz)
        elems.append(m.tets + node_off[-1])
        mats.append(rng.integers(0, 2, m.n_tets))
        fixeds.append(bnd.astype(np.uint8))
        node_off.append(node_off[-1] + m.n_nodes)
        elem_off.append(elem_off[-1] + m.n_tets)
        sizes.append(m)
    xyz = np.concatenate(xyzs)
    x0 = np.zeros((xyz.shape[0], R, 3))
    fixed = np.concatenate(fixeds)
    x0[fixed == 1] = rng.uniform(-1, 1, (int(fixed.sum()), R, 3))
    return (np.array(node_off), xyz, np.array(elem_off), np.concatenate(elems), np.concatenate(mats), fixed, x0, sizes)


def _oracle_solve(dim, node_off, xyz, elem_off, elems, mat, fixed, x0, E, nu):
    out = np.zeros_like(x0)
    for s in range(node_off.size - 1):
        a, b = node_off[s], node_off[s + 1]
        el = elems[elem_off[s]:elem_off[s + 1]] - a
        K = ocells.assemble(xyz[a:b], el, mat[elem_off[s]:elem_off[s + 1]], E, nu)
        bn = np.nonzero(fixed[a:b])[0]
        for r in range(x0.shape[1]):
            out[a:b, r] = ocells.solve_dirichlet(K, b - a, bn, x0[a:b][bn, r])
    return out


@pytest.mark.parametrize("precision", [FP64, FP32_IR])
def test_batched_volume_problems_match_oracle(lib, cuda, precision):
    E, nu = np.array([1.0, 50.0]), np.array([0.3, 0.25])
    node_off, xyz, elem_off, elems, mat, fixed, x0, _ = _volume_batch()
    B = BatchSystems(3, node_off, xyz, elem_off, elems, mat, E, nu, fixed, 8)
    x, rc = B.solve(x0, precision=precision, tol=1e-10)
    assert rc == 0
    ref = _oracle_solve(3, node_off, xyz, elem_off, elems, mat, fixed, x0, E, nu)
    assert np.abs(x - ref).max() <= SOL_TOL * np.abs(ref).max()
    np.testing.assert_array_equal(x[fixed == 1], x0[fixed == 1])
    rep = B.report()
    assert np.all(rep["rel"] <= 1e-10) and np.all(rep["outer"] >= 1)
    if precision == FP32_IR:
        assert np.all(rep["outer"] >= 2)   # FP32 inner solves need refinement to reach 1e-10


def test_batched_face_problems_match_oracle(lib, cuda):
    E, nu = np.array([1.0, 50.0]), np.array([0.3, 0.25])
    rng = np.random.default_rng(4)
    node_off, elem_off, xyzs, elems, mats, fixeds = [0], [0], [], [], [], []
    for s in range(6):
        m = meshgen.kuhn_cube(4 + s % 2)
        axis = s % 3
        faces, _ = meshgen.boundary_faces_on_plane(m, axis, 1.0)
        nodes = np.unique(faces)
        loc = -np.ones(m.n_nodes, int)
        loc[nodes] = np.arange(nodes.size)
        f_xyz = m.xyz[nodes]
        other = [a for a in range(3) if a != axis]
        border = np.any((f_xyz[:, other] < 1e-12) | (f_xyz[:, other] > 1 - 1e-12), axis=1)
        xyzs.append(f_xyz)
        elems.append(loc[faces] + node_off[-1])
        mats.append(rng.integers(0, 2, faces.shape[0]))
        fixeds.append(border.astype(np.uint8))
        node_off.append(node_off[-1] + nodes.size)
        elem_off.append(elem_off[-1] + faces.shape[0])
    node_off, elem_off = np.array(node_off), np.array(elem_off)
    xyz, elems, mat, fixed = np.concatenate(xyzs), np.concatenate(elems), np.concatenate(mats), np.concatenate(fixeds)
    x0 = np.zeros((xyz.shape[0], 4, 3))
    x0[fixed == 1] = rng.uniform(-1, 1, (int(fixed.sum()), 4, 3))
    B = BatchSystems(2, node_off, xyz, elem_off, elems, mat, E, nu, fixed, 4)
    x, rc = B.solve(x0, precision=FP32_IR, tol=1e-10)
    assert rc == 0
    ref = _oracle_solve(2, node_off, xyz, elem_off, elems, mat, fixed, x0, E, nu)
    assert np.abs(x - ref).max() <= SOL_TOL * np.abs(ref).max()


@pytest.mark.parametrize("face_material", ["zero", "cells", "default"])
def test_cell_bases_match_oracle_chain(lib, cuda, face_material):
    """Both face-material conventions against the oracle chain: "zero" (material 0 on the face and
    edge problems, the reference's construction and the default) and "cells" (their tetrahedra's
    materials); "default" sets nothing and must give the reference's convention."""
    cm = meshgen.msfem_cells(n_coarse=2, m_choices=(3, 4, 5), seed=11)
    C = Cells(cm)
    if face_material != "default":
        C.set_face_material(face_material)
    assert C.build_bases(precision=FP32_IR, tol=1e-10) == 0
    B = C.bases()
    mode = "zero" if face_material == "default" else face_material
    for c in range(cm.n_cells):
        xyz, tets, mat, box = cm.cell(c)
        want = ocells.order1_bases(xyz, tets, mat, box, cm.E, cm.nu, face_material=mode)
        got = B[cm.node_off[c]:cm.node_off[c + 1]]
        assert np.abs(got - want).max() <= SOL_TOL, (c, np.abs(got - want).max())
    rep = C.report()
    assert np.all(rep["rel"] <= 1e-10) and np.all(rep["face_rel"] <= 1e-10)


@pytest.fixture(scope="module")
def full_cells():
    # 48 cells of the 16^3 macro grid, fine resolutions drawn from {8,12,16,20}
    cm = meshgen.msfem_cells(n_coarse=16, seed=3, cells=range(0, 4096, 85))
    assert set(cm.m.tolist()) == {8, 12, 16, 20}
    return cm


def test_full_size_cells_residuals_vertices_determinism(lib, cuda, full_cells):
    """FP32 inner solves with the FP64 residual check to 1e-8 (the batch's stopping rule),
    verified independently: the oracle assembles each cell in FP64 and recomputes every
    basis's residual ||F_I - A_II x_I|| / ||F_I||."""
    cm = full_cells
    C = Cells(cm)
    assert C.build_bases(precision=FP32_IR, tol=1e-8) == 0
    B = C.bases()
    for c in range(cm.n_cells):
        xyz, tets, mat, box = cm.cell(c)
        K = ocells.assemble(xyz, tets, mat, cm.E, cm.nu)
        bnd = np.nonzero(ocells.face_masks(xyz, box))[0]
        res = ocells.residual(K, B[cm.node_off[c]:cm.node_off[c + 1]], bnd)
        assert res.max() <= 2e-8, (c, res.max())
    # the 8 bases add up to (1,1,1) up to the solve error (the reference's indefinite
    # operator makes some cells ill-conditioned, so 1e-8 in the residual is ~1e-4 here)
    assert np.abs(B.sum(axis=1) - 1.0).max() < 1e-3
    for c in range(cm.n_cells):
        xyz, _, _, box = cm.cell(c)
        mask = ocells.face_masks(xyz, box)
        for v in range(8):
            want = sum(1 << f for f in ocells.vertex_faces(v))
            node = cm.node_off[c] + np.nonzero((mask & want) == want)[0][0]
            np.testing.assert_array_equal(B[node], np.eye(8)[v][:, None] * np.ones(3))
    rep = C.report()
    assert np.all(rep["rel"] <= 1e-8) and np.all(rep["face_rel"] <= 1e-8)
    # a second build gives the same bits (fixed reduction orders, no atomics in the sums)
    assert C.build_bases(precision=FP32_IR, tol=1e-8) == 0
    np.testing.assert_array_equal(C.bases(), B)


def test_full_size_cell_matches_oracle(lib, cuda, full_cells):
    """One m = 8 cell at full resolution against the oracle chain.  Its matrix is the
    reference's indefinite one and amplifies residuals by ~1e3 here, so the batch solves
    to 1e-12 for a 1e-8 comparison of the bases."""
    cm = full_cells
    c = int(np.nonzero(cm.m == 8)[0][0])
    one = meshgen.CellMeshes(node_off=np.array([0, cm.node_off[c + 1] - cm.node_off[c]]),
                             xyz=cm.cell(c)[0], tet_off=np.array([0, cm.tet_off[c + 1] - cm.tet_off[c]]),
                             tets=cm.cell(c)[1], mat=cm.cell(c)[2], box=cm.box[c:c + 1], E=cm.E, nu=cm.nu,
                             m=cm.m[c:c + 1])
    C = Cells(one)
    assert C.build_bases(precision=FP32_IR, tol=1e-12) == 0
    xyz, tets, mat, box = one.cell(0)
    want = ocells.order1_bases(xyz, tets, mat, box, one.E, one.nu, face_material="zero")
    assert np.abs(C.bases() - want).max() <= SOL_TOL


def test_face_material_switch_round_trip(lib, cuda):
    """Switching to "cells" and back to "zero" gives the default's bases bit for bit: the switch
    restores the face batch's materials exactly."""
    cm = meshgen.msfem_cells(n_coarse=2, m_choices=(3, 4), seed=5)
    C = Cells(cm)
    assert C.build_bases(precision=FP64, tol=1e-11) == 0
    B0 = C.bases()
    C.set_face_material("cells")
    assert C.build_bases(precision=FP64, tol=1e-11) == 0
    B1 = C.bases()
    C.set_face_material("zero")
    assert C.build_bases(precision=FP64, tol=1e-11) == 0
    np.testing.assert_array_equal(C.bases(), B0)
    assert np.abs(B1 - B0).max() > 1e-6      # the inclusions make the conventions differ


def test_order1_bases_and_driver_match_reference_run(lib, cuda):
    """The reference's own whole Order1 run (tests/golden/msfem_order1.npz, made by oracle/_ref's
    order2_ref --order1 from MsFEM::MsFEM_forElasticDeformation_OrderBF1_forPoly, MsFEM/MsFEM.h:
    572-1010, on graded cells with inclusions): the GPU bases of cells 0 and 7 within 1e-8 of the
    reference's, and the GPU Order1 driver's macro solution within 1e-8 relative L2 of its."""
    import os
    import types

    from multiscalefemsolver3d_b200.msfem import msfem_elastic_driver
    from oracle import order2 as o2
    d = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "msfem_order1.npz"))
    vxyz, cv, cm = o2.graded_cells(2, 4, 0.5)
    assert abs(cm.xyz.sum() - float(d["xyz_sum"])) < 1e-9
    C = Cells(cm)
    assert C.build_bases(precision=FP64, tol=1e-12) == 0
    B = C.bases()
    for c in (0, 7):
        got = B[cm.node_off[c]:cm.node_off[c + 1]]
        assert np.abs(got - d[f"bases_{c}"]).max() <= SOL_TOL, (c, np.abs(got - d[f"bases_{c}"]).max())
    bot = np.nonzero(np.abs(vxyz[:, 2]) < 1e-12)[0]
    top = np.nonzero(np.abs(vxyz[:, 2] - 1) < 1e-12)[0]
    fv = np.concatenate([bot, top]).astype(np.int32)
    vals = np.concatenate([np.zeros((bot.size, 3)), np.tile([0.01, -0.02, 0.05], (top.size, 1))])
    cc = types.SimpleNamespace(cells=cm, cell_vertex=cv, n_coarse_vertices=vxyz.shape[0])
    res = msfem_elastic_driver(cc, fv, vals, np.zeros((0, 2), np.int32), np.zeros((0, 3)), precision=FP64,
                               tol=1e-13, cell_tol=1e-12, cells=C)
    assert np.linalg.norm(res.U - d["solution"]) <= 1e-8 * np.linalg.norm(d["solution"])


def test_cells_reject_bad_meshes(lib, cuda):
    cm = meshgen.msfem_cells(n_coarse=2, m_choices=(3,), seed=1, cells=[0, 1])
    bad = meshgen.CellMeshes(**{k: getattr(cm, k).copy() for k in cm.__dataclass_fields__})
    bad.tets[5, 2] = 10_000                       # node id outside its cell
    with pytest.raises(_lib.MsfemError) as e:
        Cells(bad)
    assert e.value.rc == _lib.MSFEM_ERR_ARGUMENT
    bad = meshgen.CellMeshes(**{k: getattr(cm, k).copy() for k in cm.__dataclass_fields__})
    bad.box[1, 1] += 0.01                         # box corner without a node
    with pytest.raises(_lib.MsfemError) as e:
        Cells(bad)
    assert e.value.rc == _lib.MSFEM_ERR_ARGUMENT


def test_macro_element_matrices_match_oracle(lib, cuda):
    cm = meshgen.msfem_cells(n_coarse=2, m_choices=(3, 4, 5), seed=11)
    C = Cells(cm)
    assert C.build_bases(precision=FP32_IR, tol=1e-10) == 0
    B = C.bases()
    K = C.macro_matrices()
    for c in range(cm.n_cells):
        xyz, tets, mat, box = cm.cell(c)
        want = ocells.macro_element_matrix(xyz, tets, B[cm.node_off[c]:cm.node_off[c + 1]], box, cm.E[0], cm.nu[0])
        np.testing.assert_allclose(K[c], want, rtol=0, atol=1e-12 * np.abs(want).max())


def test_full_size_macro_matrices_translation_free(lib, cuda, full_cells):
    cm = full_cells
    C = Cells(cm)
    assert C.build_bases(precision=FP32_IR, tol=1e-8) == 0
    K = C.macro_matrices()
    np.testing.assert_allclose(K, K.transpose(0, 2, 1, 4, 3), rtol=0, atol=1e-13 * np.abs(K).max())
    f = np.einsum("cijrs,s->cir", K, np.array([1.0, 1.0, 1.0]))
    # the bases add up to (1,1,1) to the solve's accuracy (ill-conditioned cells: ~1e-4 here)
    assert np.abs(f).max() <= 1e-3 * np.abs(K).max()


def test_build_graph_replay_is_bit_identical(lib, cuda):
    """The first build runs launch by launch (and tunes the persistent launches' CTA sizes), the
    second is captured into a CUDA graph, the third replays it: the same bases, bit for bit, and
    the oracle chain's within 1e-8; changing the face materials between replays changes values in
    place, which the replayed graph picks up."""
    cm = meshgen.msfem_cells(n_coarse=2, m_choices=(3, 4, 5), seed=11)
    C = Cells(cm)
    out = []
    for _ in range(3):
        assert C.build_bases(precision=FP32_IR, tol=1e-10) == 0
        out.append(C.bases())
    np.testing.assert_array_equal(out[0], out[1])
    np.testing.assert_array_equal(out[0], out[2])
    C.set_face_material("cells")
    assert C.build_bases(precision=FP32_IR, tol=1e-10) == 0
    B = C.bases()
    for c in range(cm.n_cells):
        xyz, tets, mat, box = cm.cell(c)
        want = ocells.order1_bases(xyz, tets, mat, box, cm.E, cm.nu, face_material="cells")
        assert np.abs(B[cm.node_off[c]:cm.node_off[c + 1]] - want).max() <= SOL_TOL
