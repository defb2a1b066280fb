"""The MsFEM Order2 restatement (oracle/order2.py) against the reference's own Order2 construction
run here: oracle/_ref/order2_ref calls MsFEM::Grid_forMech::Initialization (topology and
CreateFunctionalSpaces, MsFEM/MsFEM_Grid.h:1001-3080) and the macro element's SolveLocalMatrix on
a macro mesh and cell directories written by meshio."""
import os

import numpy as np
import pytest

from oracle import order2 as o2

pytestmark = pytest.mark.skipif(not os.path.exists(o2.ORDER2_REF),
                                reason="oracle/_ref/order2_ref not built (make -C oracle ref)")


def test_order2_bases_and_macro_matrix_match_reference(tmp_path):
    """A graded 8^3 cell with inclusions (E 1:10): the 27 bases within 1e-11 of the reference's
    BasisFunction files, the 81 x 81 macro element matrix within 1e-11 of its SolveLocalMatrix."""
    vxyz, cv, cm = o2.graded_cells(1, 8, 0.5)
    R = o2.run_reference(str(tmp_path), vxyz, cv, cm)
    xyz, tets, mat, box = cm.cell(0)
    assert 0 < mat.sum() < mat.size
    ours = o2.order2_bases(xyz, tets, mat, box, cm.E, cm.nu, cv[0])
    ref = R["bases"][0]
    np.testing.assert_allclose(ours, ref, rtol=0, atol=1e-11 * np.abs(ref).max())
    K = o2.macro_element_matrix(xyz, tets, ours, box, cm.E[0], cm.nu[0])
    np.testing.assert_allclose(K.transpose(0, 2, 1, 3).reshape(81, 81), R["K"][0], rtol=0,
                               atol=1e-11 * np.abs(R["K"][0]).max())
    # the face problems get no load (FEM_2D adds it only when it logs): face bubbles vanish on
    # their face; every bubble vanishes at the cell vertices
    mask = o2.oc.face_masks(xyz, box)
    for f in range(6):
        np.testing.assert_array_equal(ref[((mask >> f) & 1).astype(bool), 20 + f], 0.0)
    corners = np.array([np.nonzero(np.all(np.abs(xyz - v) < 1e-12, axis=1))[0][0]
                        for v in o2.oc.box_vertices(box)])
    np.testing.assert_allclose(ref[corners][:, :8], np.repeat(np.eye(8)[:, :, None], 3, axis=2), atol=1e-13)
    np.testing.assert_array_equal(ref[corners][:, 8:], 0.0)


def test_order2_topology_and_dof_numbering(tmp_path):
    """2 x 2 x 2 cells: edges, faces, each face's edges and each cell's 27 DOF ids as the
    reference's CreateTopology and CreateFunctionalSpaces number them."""
    vxyz, cv, cm = o2.graded_cells(2, 1, 0.0)
    R = o2.run_reference(str(tmp_path), vxyz, cv, cm, matrices=False)
    edges, faces, cell_faces, dofs = o2.macro_topology(cv)
    assert list(R["n"]) == [8, 27, len(edges), len(faces), 27 + len(edges) + len(faces) + 8]
    np.testing.assert_array_equal(R["edges"], edges)
    np.testing.assert_array_equal(R["cell_faces"], cell_faces)
    np.testing.assert_array_equal(R["cell_dofs"], dofs)
    eid = {tuple(p): i for i, p in enumerate(edges)}
    rec, i = R["faces"], 0
    while i < rec.size:
        f, k = rec[i], rec[i + 1]
        cyc = faces[f]
        want = [eid[(min(cyc[j], cyc[(j + 1) % 4]), max(cyc[j], cyc[(j + 1) % 4]))] for j in range(4)]
        np.testing.assert_array_equal(rec[i + 2:i + 2 + k], want)
        i += 2 + k


def test_reference_loses_uniform_edge_solutions(tmp_path):
    """On uniform segments the reference's edge solves meet MIN_RESIDUAL = 1e-15 on their first
    pass and the restart loop returns the initial guess (FEM/FEM.h:3704-3771): its vertex bases
    are 0 inside the cell edges, where the converged edge solution is linear.  The restatement
    keeps the converged solution."""
    vxyz, cv, cm = o2.graded_cells(1, 3, 0.0)
    R = o2.run_reference(str(tmp_path), vxyz, cv, cm, matrices=False)
    xyz, tets, mat, box = cm.cell(0)
    ours = o2.order2_bases(xyz, tets, mat, box, cm.E, cm.nu, cv[0])
    on = (np.abs(xyz[:, 1]) < 1e-12) & (np.abs(xyz[:, 2]) < 1e-12)        # the edge from vertex 0 to 1
    nodes = np.nonzero(on)[0][np.argsort(xyz[on, 0])]
    np.testing.assert_array_equal(R["bases"][0][nodes[1:-1], 0], 0.0)
    np.testing.assert_allclose(ours[nodes, 0, 0], [1, 2 / 3, 1 / 3, 0], atol=1e-14)


def test_order2_driver_matches_reference(tmp_path):
    """The whole Order2 driver (MsFEM_forElasticDeformation_OrderBF2_forPoly) on 2 x 2 x 2 graded
    cells with inclusions, u = 0 on z = 0 and u = (0.01, -0.02, 0.05) on z = 1: the macro solution
    of the restated driver (own bases, L2-projected Dirichlet values, row and column elimination,
    exact solve) within 1e-9 of the reference's (plain CG restarts to 1e-13).  The Dirichlet faces'
    bubble DOFs come out 0 and their edge DOFs ~0: the vertex bases alone carry a constant."""
    vxyz, cv, cm = o2.graded_cells(2, 4, 0.5)
    bot = np.nonzero(np.abs(vxyz[:, 2]) < 1e-12)[0]
    top = np.nonzero(np.abs(vxyz[:, 2] - 1) < 1e-12)[0]
    groups = [(bot, (0.0, 0.0, 0.0), (1, 1, 1)), (top, (0.01, -0.02, 0.05), (1, 1, 1))]
    R = o2.run_reference(str(tmp_path), vxyz, cv, cm, matrices=False, groups=groups, min_residual=1e-13)
    ref = R["solution"]
    x = o2.order2_driver(vxyz, cv, cm, groups)
    assert np.linalg.norm(x - ref) <= 1e-9 * np.linalg.norm(ref)
    np.testing.assert_allclose(ref[top], np.tile([0.01, -0.02, 0.05], (top.size, 1)), atol=1e-15)
    edges, faces, _, _ = o2.macro_topology(cv)
    nv, ne = vxyz.shape[0], len(edges)
    top_faces = [nv + ne + i for i in range(len(faces)) if set(faces[i]) <= set(top)]
    np.testing.assert_array_equal(ref[top_faces], 0.0)


def test_order2_macro_portrait_matches_reference(tmp_path, lib):
    """The restatement's portrait rule (o2.macro_portrait: the DOFs sharing a cell; the GPU macro
    system is checked against it in tests/test_gpu_order2.py) is the reference driver's block
    portrait: per DOF row, the columns below and above the diagonal (CreationPortrait)."""
    vxyz, cv, cm = o2.graded_cells(2, 1, 0.0)
    top = np.nonzero(np.abs(vxyz[:, 2] - 1) < 1e-12)[0]
    R = o2.run_reference(str(tmp_path), vxyz, cv, cm, matrices=False,
                         groups=[(top, (0.0, 0.0, 0.01), (1, 1, 1))], min_residual=1e-12)
    edges, faces, _, dofs = o2.macro_topology(cv)
    n_dofs = vxyz.shape[0] + len(edges) + len(faces) + len(cv)
    rule = o2.macro_portrait(dofs, n_dofs)
    rec, i = R["portrait"], 0
    for d in range(n_dofs):
        nd = rec[i]
        down = rec[i + 1:i + 1 + nd]
        i += 1 + nd
        nu = rec[i]
        up = rec[i + 1:i + 1 + nu]
        i += 1 + nu
        np.testing.assert_array_equal(rule[d], np.concatenate([np.sort(down), [d], np.sort(up)]))
    assert i == rec.size
