"""The reference's mesh files (multiscalefemsolver3d_b200/meshio.py): what this package writes,
the reference's own readers (math::SimpleGrid::ReadFromNVTR / ReadFromSalomeDat, compiled from
its sources in oracle/_ref) read back identically, and this package's readers follow the same
rules: 1-based ids unless a 0 appears, the dropped last element of a file that ends right after
a digit, polyhedral records, Salome vertex maps."""
import os

import numpy as np
import pytest

from multiscalefemsolver3d_b200 import meshgen, meshio


def _mesh(n=3, seed=0):
    m = meshgen.kuhn_cube(n, jitter=0.1, seed=seed)
    m.mat[:] = np.random.default_rng(seed).integers(0, 3, m.n_tets)
    return m


@pytest.mark.parametrize("one_based", [True, False])
def test_nvtr_round_trip_and_reference_reader(tmp_path, ref, one_based):
    m = _mesh()
    d = tmp_path / "mesh"
    meshio.write_nvtr(d, m.xyz, m.tets, m.mat, one_based=one_based)
    xyz, el, kat, rfz = meshio.read_nvtr(d, 4)
    np.testing.assert_array_equal(xyz, m.xyz)
    np.testing.assert_array_equal(el, m.tets)
    np.testing.assert_array_equal(kat, m.mat)
    assert rfz == (not one_based)
    rx, rel, rkat, rrfz = ref.read_nvtr(d, 4, m.n_nodes, m.n_tets, 4 * m.n_tets)
    np.testing.assert_array_equal(rx, m.xyz)
    np.testing.assert_array_equal(np.array(rel), m.tets)
    np.testing.assert_array_equal(rkat, m.mat)
    assert rrfz == rfz


def test_one_based_polyhedra_are_refused(tmp_path):
    """The reference's reader corrupts 1-based polyhedral records (an inner `ii` shadows the
    outer one, Math.h:241-256); this reader refuses them instead of guessing."""
    d = tmp_path / "poly"
    rec = np.array([4, 1, 2, 3, 4, 1, 3, 1, 2, 3])
    meshio.write_nvtr(d, np.zeros((4, 3)), [rec - np.array([0, 1, 1, 1, 1, 0, 0, 1, 1, 1])], one_based=True)
    with pytest.raises(ValueError, match="1-based polyhedral"):
        meshio.read_nvtr(d, -1)


def test_nvtr_without_trailing_newline_loses_its_last_element(tmp_path, ref):
    m = _mesh(2, seed=1)
    d = tmp_path / "mesh"
    meshio.write_nvtr(d, m.xyz, m.tets, m.mat)
    p = d / "nvtr.txt"
    p.write_bytes(p.read_bytes().rstrip(b"\n"))
    xyz, el, kat, rfz = meshio.read_nvtr(d, 4)
    assert el.shape[0] == m.n_tets - 1
    _, rel, rkat, rrfz = ref.read_nvtr(d, 4, m.n_nodes, m.n_tets, 4 * m.n_tets)
    assert len(rel) == m.n_tets - 1
    np.testing.assert_array_equal(np.array(rel), el)
    np.testing.assert_array_equal(rkat, kat)


def test_macro_polyhedra_and_cell_directories(tmp_path, ref):
    m = meshgen.kuhn_cube(4)
    cc = meshgen.cube_cells(m, np.array([1.0]), np.array([0.3]), 2)
    nc = round(cc.cells.n_cells ** (1 / 3))
    g = np.arange(nc + 1) / nc
    kk, jj, ii = np.meshgrid(g, g, g, indexing="ij")
    vxyz = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], axis=1)
    d = tmp_path / "macro"
    meshio.write_macro_nvtr(d, vxyz, cc.cell_vertex)
    xyz, recs, kat, rfz = meshio.read_nvtr(d, -1)
    assert rfz and len(recs) == cc.cells.n_cells       # polyhedra are written 0-based
    np.testing.assert_array_equal(recs[0][1:9], cc.cell_vertex[0])
    # face cycles in the cell's local vertex numbers
    np.testing.assert_array_equal(recs[0][10:].reshape(6, 5)[:, 1:], meshio.FACE_CYCLES)
    rx, rrecs, rkat, rrfz = ref.read_nvtr(d, -1, vxyz.shape[0], cc.cells.n_cells, 40 * cc.cells.n_cells)
    assert rrfz == rfz
    for a, b in zip(recs, rrecs):
        np.testing.assert_array_equal(a, b)
    root = tmp_path / "cells"
    meshio.write_cell_dirs(root, cc.cells)
    for c in (0, cc.cells.n_cells - 1):
        sub = root / f"Elem_{c}" / "SubElem_0"
        cx, ct, cm, cb = cc.cells.cell(c)
        xyz, el, kat, _ = meshio.read_nvtr(sub, 4)
        np.testing.assert_array_equal(el, ct)
        for f in range(6):
            fx, fe, fmap = meshio.read_salome_dat(sub / f"Face_id{f}.dat", 2, with_map=True)
            rx, re, rmap = ref.read_salome(sub / f"Face_id{f}.dat", 2, cx.shape[0], 1000, 1000)
            np.testing.assert_array_equal(fx, rx)
            np.testing.assert_array_equal(fe, re)
            np.testing.assert_array_equal(fmap, rmap)
            # the map takes the face's vertices to the cell's own nodes, all on face f
            axis, side = f // 2, f % 2
            np.testing.assert_allclose(cx[fmap, axis], cb[2 * axis + side], atol=1e-15)
            # elements name the cell's own node ids, each a tet face on face f
            assert set(np.unique(fe)) <= set(fmap)
            np.testing.assert_allclose(cx[fe, axis], cb[2 * axis + side], atol=1e-15)
            assert fe.shape[0] == 2 * cc.cells.m[c] ** 2


def test_kraev_round_trip(tmp_path):
    lists = [np.array([0, 5, 7]), np.array([], dtype=np.int64), np.array([3, 2])]
    p = tmp_path / "kraev1.txt"
    meshio.write_kraev(p, lists, one_based=True)
    back = meshio.read_kraev(p, 3, read_from_zero=False)
    for a, b in zip(lists, back):
        np.testing.assert_array_equal(a, b)
    assert p.read_text().split()[0] == "5"
