"""Host logic of the Order2 GPU path, checked without a GPU: the edge-basis order the library
derives from the cells' global vertex ids is the reference's edge numbering as the restatement
(oracle/order2.py, pinned against the reference's topology) orders it."""
import numpy as np
import pytest

from multiscalefemsolver3d_b200 import cells as gcells
from oracle import order2 as o2


def _edge_info(e):
    axis, s, t = e // 4, (e >> 1) & 1, e & 1
    o0, o1 = (1 if axis == 0 else 0), (1 if axis == 2 else 2)
    vl = (s << o0) | (t << o1)
    return vl, vl | (1 << axis)


def test_order2_edge_order_matches_restatement(lib):
    rng = np.random.default_rng(0)
    cv = np.array([rng.permutation(50)[:8] for _ in range(40)], np.int32)
    _, cv_grid, _ = o2.graded_cells(2, 1, 0.0)
    cv = np.concatenate([cv, cv_grid.astype(np.int32)])
    got = gcells.order2_edge_order(cv)
    for c in range(cv.shape[0]):
        topo = o2._Topo(cv[c])
        for k, e in enumerate(got[c]):
            vl, vh = _edge_info(int(e))
            assert set(topo.edges[k]) == {vl, vh}


def test_order2_edge_order_rejects_repeated_vertices(lib):
    with pytest.raises(Exception):
        gcells.order2_edge_order(np.array([[0, 1, 2, 3, 4, 5, 6, 6]], np.int32))


def _case():
    vxyz, cv, cm = o2.graded_cells(2, 3, 0.4)
    bases = []
    for c in range(cm.n_cells):
        xyz, tets, mat, box = cm.cell(c)
        bases.append(o2.order2_bases(xyz, tets, mat, box, cm.E, cm.nu, cv[c]))
    bot = np.nonzero(np.abs(vxyz[:, 2]) < 1e-12)[0]
    top = np.nonzero(np.abs(vxyz[:, 2] - 1) < 1e-12)[0]
    side = np.nonzero(np.abs(vxyz[:, 0] - 1) < 1e-12)[0]
    groups = [(bot, (0.0, 0.0, 0.0), (1, 1, 1)), (top, (0.01, -0.02, 0.05), (1, 1, 1)),
              (side, (0.03, 0.0, 0.0), (1, 0, 0))]
    return vxyz, cv, cm, bases, groups


def _expected_projection(lay, groups, want):
    """The restatement's fixed list [(scalar DOF, value)] read back into the layout's [group DOF
    k][c] slots: entry j of the list is the j-th (group, k, taken c) in the layout's order, so its
    DOF must be 3 gd[k] + c."""
    P = np.full(3 * lay.group_dofs.size, np.nan)
    j = 0
    for g, (_, _, take) in enumerate(groups):
        for k in range(lay.group_dof_off[g], lay.group_dof_off[g + 1]):
            for comp in range(3):
                if take[comp]:
                    assert want[j][0] == 3 * int(lay.group_dofs[k]) + comp
                    P[3 * k + comp] = want[j][1]
                    j += 1
    assert j == len(want)
    return P


def test_order2_topology_and_dirichlet_layout_match_restatement(lib):
    """The product's host side of the Order2 driver (macro topology, the groups' DOF and face
    lists, the elimination order) against the restatement (oracle/order2.py, pinned against the
    reference's topology and whole driver): the same topology; per group the restatement's DOFs in
    its order, its faces with their 9 DOFs; and the rows eliminated, with the restatement's
    projected values gathered through the layout, give the restated driver's solution.  (The
    projection itself, the macro system and the solve run on the GPU: tests/test_gpu_order2.py.)"""
    from multiscalefemsolver3d_b200 import order2 as p2
    vxyz, cv, cm, bases, groups = _case()
    topo = p2.macro_topology(cv, n_vertices=vxyz.shape[0])
    edges, faces, cell_faces, dofs = o2.macro_topology(cv)
    np.testing.assert_array_equal(topo.edges, edges)
    np.testing.assert_array_equal(topo.faces, faces)
    np.testing.assert_array_equal(topo.cell_faces, cell_faces)
    np.testing.assert_array_equal(topo.cell_dofs, dofs)
    lay = p2.dirichlet_layout(topo, groups)
    nv, ne = vxyz.shape[0], len(edges)
    eid = {tuple(e): i for i, e in enumerate(edges)}
    for g, (verts, _, _) in enumerate(groups):
        sv = set(int(v) for v in verts)
        tf = [i for i in range(len(faces)) if set(int(v) for v in faces[i]) <= sv]
        rows = lay.faces[lay.group_face_off[g]:lay.group_face_off[g + 1]]
        assert len(rows) == len(tf)
        for r, f in zip(rows, tf):
            cyc = [int(v) for v in faces[f]]
            fd = cyc + [nv + eid[(min(cyc[k], cyc[(k + 1) % 4]), max(cyc[k], cyc[(k + 1) % 4]))] for k in range(4)]
            assert list(r[1:]) == fd + [nv + ne + f]
            assert f in cell_faces[r[0]]
    want = o2.dirichlet_fixed(vxyz, cv, cm, groups, bases)
    P = _expected_projection(lay, groups, want)
    last = {}
    for i, v in want:
        last[i] = v
    np.testing.assert_array_equal(lay.fixed_dofs, list(last.keys()))
    np.testing.assert_array_equal(P[lay.fixed_src], list(last.values()))
    # the composition: the dense macro system, the layout's eliminations, the restated driver, on
    # groups without shared DOFs (the product eliminates a shared row once, with its last value)
    groups = groups[:2]
    lay = p2.dirichlet_layout(topo, groups)
    P = _expected_projection(lay, groups, o2.dirichlet_fixed(vxyz, cv, cm, groups, bases))
    n = 3 * topo.n_dofs
    M = np.zeros((n, n))
    for c in range(cm.n_cells):
        K = o2.macro_element_matrix(*cm.cell(c)[:2], bases[c], cm.cell(c)[3], cm.E[0], cm.nu[0])
        idx = (3 * dofs[c][:, None] + np.arange(3)).ravel()
        M[np.ix_(idx, idx)] += K.transpose(0, 2, 1, 3).reshape(81, 81)
    F = np.zeros(n)
    for i, s in zip(lay.fixed_dofs, lay.fixed_src):
        v = P[s]
        col = M[:, i].copy()
        col[i] = 0.0
        F -= col * v
        M[:, i] = 0.0
        M[i, :] = 0.0
        M[i, i] = 1.0
        F[i] = v
    x = np.linalg.solve(M, F).reshape(-1, 3)
    xo = o2.order2_driver(vxyz, cv, cm, groups, bases=bases)
    assert np.linalg.norm(x - xo) <= 1e-11 * np.linalg.norm(xo)


def test_order2_layout_rejects_shared_faces(lib):
    """A group holding an interior face (shared by two cells) is refused, as the restatement
    assumes every Dirichlet face lies on the boundary."""
    from multiscalefemsolver3d_b200 import order2 as p2
    vxyz, cv, cm = o2.graded_cells(2, 1, 0.0)
    topo = p2.macro_topology(cv, n_vertices=vxyz.shape[0])
    mid = np.nonzero(np.abs(vxyz[:, 2] - 0.5) < 1e-12)[0]
    with pytest.raises(ValueError):
        p2.dirichlet_layout(topo, [(mid, (0.0, 0.0, 0.0), (1, 1, 1))])


def test_order2_layout_of_a_group_without_faces(lib):
    """A Dirichlet group holding no whole face (one vertex; an edge's two vertices): its DOF list is
    the vertices and edges it holds, it has no faces -- so its projection matrix is empty and the
    projected values are 0, as the restatement's least-squares solve gives -- and its taken
    components are still eliminated, in order."""
    from multiscalefemsolver3d_b200 import order2 as p2
    vxyz, cv, cm = o2.graded_cells(2, 1, 0.0)
    topo = p2.macro_topology(cv, n_vertices=vxyz.shape[0])
    a, b = (int(v) for v in topo.edges[0])
    groups = [([a], (0.1, 0.2, 0.3), (1, 0, 1)), ([a, b], (0.0, 0.0, 0.0), (0, 1, 0))]
    lay = p2.dirichlet_layout(topo, groups)
    assert lay.faces.shape == (0, 10)
    np.testing.assert_array_equal(lay.group_face_off, [0, 0, 0])
    nv = topo.n_vertices
    np.testing.assert_array_equal(lay.group_dofs, [a, min(a, b), max(a, b), nv + 0])
    np.testing.assert_array_equal(lay.group_dof_off, [0, 1, 4])
    # rows: group 0 takes x and z of a; group 1 takes y of a, b and the edge
    want_rows = [3 * a, 3 * a + 2] + [3 * d + 1 for d in sorted([a, b])] + [3 * (nv + 0) + 1]
    np.testing.assert_array_equal(lay.fixed_dofs, want_rows)
    np.testing.assert_array_equal(lay.fixed_src, [0, 2] + [3 * k + 1 for k in (1, 2, 3)])
