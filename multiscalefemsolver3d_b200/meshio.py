"""The reference's mesh and boundary files, read and written on the host.

The reference reads every mesh from text files (Library/Math.h:26-291, FEM/FEM_Main.cpp,
MsFEM/MsFEM_Main.cpp); these functions write the synthetic workloads in those formats, so that
the reference's own executables can run on the same inputs, and read them back with the
reference's rules:

* NVTR directory (`math::SimpleGrid::ReadFromNVTR`, Math.h:150-291): `param.txt` = "n_vertices
  n_elements", `xyz.txt` = 3 coordinates per vertex, `nvtr.txt` = the vertex ids of each element
  (k per element, or for polyhedra `n v_1..v_n n_faces (m w_1..w_m)...`), `nvkat.txt` = the
  material of each element (optional: zeros when absent).  Ids are 1-based unless some id is 0
  (then 0-based: `read_from_zero`).  Quirk reproduced: an element is kept only if the file does
  not end right after its last digit (`feof` after the `fscanf`), so a file without a trailing
  newline loses its last element.  Quirk avoided: the reference's 1-based shift of polyhedral
  records (Math.h:241-256) declares a second `ii` inside its `for`, so it reads the face count
  from the record's first entry and indexes past the record -- a 1-based polyhedral file crashes
  it.  Polyhedra are therefore written 0-based, and read_nvtr refuses 1-based ones.
* Boundary lists `kraev1.txt` / `kraev2.txt` (FEM/FEM_Main.cpp:693-714, :800-821): "N" then N
  pairs "vertex type", shifted by -1 when the mesh was 1-based.
* Salome `.dat` (`ReadFromSalomeDat`, Math.h:35-149): "n_vertices n_elements", vertex lines
  "id x y z", element lines "id type v..." with type 102 / 203 / 304 (segment / triangle / tet),
  1-based; with a map, vertex_map[i] = id_i - 1 (the face files of the MsFEM cells use the cell's
  own node ids there).
* MsFEM cell directories (MsFEM/MsFEM_Grid.h:4837-4850): `<root>/Elem_<c>/SubElem_0` holds cell
  c's fine mesh as NVTR, and `Face_id<f>.dat` its face f's triangles in Salome format with the
  cell's node ids as vertex ids; the macro mesh is an NVTR directory of polyhedra.
"""
from __future__ import annotations

import os

import numpy as np

from .meshgen import CellMeshes

__all__ = ["write_nvtr", "read_nvtr", "write_kraev", "read_kraev", "write_salome_dat", "read_salome_dat",
           "write_cell_dirs", "write_macro_nvtr", "write_tecplot", "elastic_result_fields"]


def _ints_text(rows) -> str:
    return "".join(" ".join(str(int(v)) for v in r) + "\n" for r in rows)


def write_nvtr(directory, xyz, elems, mat=None, one_based=True):
    """elems: [n, k] ints, or a list of flattened polyhedron records (see module docstring)."""
    os.makedirs(directory, exist_ok=True)
    xyz = np.asarray(xyz, dtype=np.float64)
    off = 1 if one_based else 0
    if isinstance(elems, np.ndarray):
        rows = np.asarray(elems, dtype=np.int64) + off
    else:
        rows = [_shift_poly(np.asarray(r, dtype=np.int64), off) for r in elems]
    n = len(rows)
    with open(os.path.join(directory, "param.txt"), "w") as f:
        f.write(f"{xyz.shape[0]} {n}\n")
    with open(os.path.join(directory, "xyz.txt"), "w") as f:
        f.write("".join(f"{x:.17g} {y:.17g} {z:.17g}\n" for x, y, z in xyz))
    with open(os.path.join(directory, "nvtr.txt"), "w") as f:
        f.write(_ints_text(rows))
    if mat is not None:
        with open(os.path.join(directory, "nvkat.txt"), "w") as f:
            f.write("".join(f"{int(m)}\n" for m in np.asarray(mat)))


def _shift_poly(rec, off):
    """Adds `off` to the vertex ids of a flattened polyhedron record, leaving the counts."""
    out = rec.copy()
    i = 0
    n = int(rec[i])
    out[1:1 + n] += off
    i = 1 + n
    nf = int(rec[i])
    i += 1
    for _ in range(nf):
        m = int(rec[i])
        out[i + 1:i + 1 + m] += off
        i += 1 + m
    return out


def _poly_len(tokens, i):
    """Number of tokens of the polyhedron record starting at tokens[i] (None if truncated)."""
    j = i
    if j >= len(tokens):
        return None
    n = int(tokens[j])
    j += 1 + n
    if j >= len(tokens):
        return None
    nf = int(tokens[j])
    j += 1
    for _ in range(nf):
        if j >= len(tokens):
            return None
        j += 1 + int(tokens[j])
    return j - i if j <= len(tokens) else None


def read_nvtr(directory, k):
    """(xyz [nv, 3], elems ([ne, k] int array, or a list of polyhedron records for k = -1), nvkat
    [ne], read_from_zero) with the reference reader's rules (module docstring)."""
    with open(os.path.join(directory, "param.txt")) as f:
        nv, ne = (int(t) for t in f.read().split()[:2])
    xyz = np.fromfile(os.path.join(directory, "xyz.txt"), sep=" ")[:3 * nv].reshape(-1, 3)
    with open(os.path.join(directory, "nvtr.txt"), "rb") as f:
        raw = f.read()
    tokens = raw.split()
    ends_in_digit = len(raw) > 0 and raw[-1:].isdigit()
    elems, i = [], 0
    for e in range(ne):
        n_tok = k if k > 0 else _poly_len(tokens, i)
        if n_tok is None or i + n_tok > len(tokens):
            break
        rec = [int(t) for t in tokens[i:i + n_tok]]
        i += n_tok
        if i == len(tokens) and ends_in_digit:   # fscanf hit the end of the file: feof drops it
            break
        elems.append(rec)
    if k > 0:
        flat = np.array(elems, dtype=np.int64).reshape(-1, k)
        read_from_zero = bool((flat == 0).any())
        if not read_from_zero:
            flat = flat - 1
        out = flat
    else:
        read_from_zero = any(0 in r for r in elems)
        if not read_from_zero and elems:
            raise ValueError("1-based polyhedral NVTR: the reference's reader mis-shifts these (Math.h:241-256); "
                             "write polyhedra 0-based")
        out = [np.asarray(r, dtype=np.int64) for r in elems]
    nk = len(elems)
    kat_path = os.path.join(directory, "nvkat.txt")
    if os.path.exists(kat_path):
        kat = np.fromfile(kat_path, sep=" ").astype(np.int64)[:nk]
        kat = np.concatenate([kat, np.zeros(nk - kat.size, np.int64)])
    else:
        kat = np.zeros(nk, np.int64)
    return xyz, out, kat, read_from_zero


def write_kraev(path, vertices_by_type, one_based=True):
    """vertices_by_type: list (type t) of vertex-id arrays -> "N" + "vertex type" lines."""
    off = 1 if one_based else 0
    pairs = [(int(v) + off, t) for t, vs in enumerate(vertices_by_type) for v in np.asarray(vs)]
    with open(path, "w") as f:
        f.write(f"{len(pairs)}\n" + "".join(f"{v} {t}\n" for v, t in pairs))


def read_kraev(path, n_types, read_from_zero):
    """Vertex lists per type, as FEM/FEM_Main.cpp:693-714 fills them."""
    tok = np.fromfile(path, sep=" ").astype(np.int64)
    n = int(tok[0])
    pairs = tok[1:1 + 2 * n].reshape(-1, 2)
    out = [[] for _ in range(n_types)]
    for v, t in pairs:
        out[int(t)].append(int(v) if read_from_zero else int(v) - 1)
    return [np.array(o, dtype=np.int64) for o in out]


_TYPES = {2: 102, 3: 203, 4: 304}


def write_salome_dat(path, xyz, elems, vertex_ids=None):
    """Vertices numbered vertex_ids (default 1..n) and elements of 2, 3 or 4 vertices given by
    their 0-based position in xyz.  Element lines name their vertices by those vertex ids, as the
    format does: the reader keeps them (minus one) and maps them back to positions through
    vertex_map (SimpleGrid::TransferIdGlobalIntoSelf, Library/Math.h:983-991; the MsFEM grids
    renumber their face meshes that way, MsFEM/MsFEM_Grid.h:1126-1135)."""
    xyz = np.asarray(xyz, dtype=np.float64)
    elems = np.asarray(elems, dtype=np.int64)
    ids = np.arange(1, xyz.shape[0] + 1) if vertex_ids is None else np.asarray(vertex_ids, dtype=np.int64)
    typ = _TYPES[elems.shape[1]]
    lines = [f"{xyz.shape[0]} {elems.shape[0]}\n"]
    lines += [f"{int(i)} {x:.17g} {y:.17g} {z:.17g}\n" for i, (x, y, z) in zip(ids, xyz)]
    lines += [f"{e + 1} {typ} " + " ".join(str(int(ids[v])) for v in row) + "\n" for e, row in enumerate(elems)]
    with open(path, "w") as f:
        f.write("".join(lines))


def read_salome_dat(path, dim, with_map=False):
    """(xyz, elements [ne, dim + 1], vertex_map or None) as ReadFromSalomeDat returns them: the
    elements name vertex ids minus one (vertex_map values, not positions); element lines of
    another type than 102/203/304 are skipped."""
    with open(path) as f:
        tok = f.read().split()
    nv, ne = int(tok[0]), int(tok[1])
    i = 2
    xyz, vmap = np.empty((nv, 3)), np.empty(nv, np.int64)
    for v in range(nv):
        vmap[v] = int(tok[i]) - 1
        xyz[v] = [float(t) for t in tok[i + 1:i + 4]]
        i += 4
    width = {102: 2, 203: 3, 304: 4}
    elems = []
    for _ in range(ne):
        typ = int(tok[i + 1])
        i += 2
        if typ in width:
            w = width[typ]
            row = [int(t) - 1 for t in tok[i:i + w]] + [0] * (dim + 1 - w)
            elems.append(row[:dim + 1])
            i += w
    return xyz, np.array(elems, dtype=np.int64).reshape(-1, dim + 1), (vmap if with_map else None)


# faces 0..5 = x0, x1, y0, y1, z0, z1 of a box cell, as vertex cycles of its corners
FACE_CYCLES = [[0, 2, 6, 4], [1, 3, 7, 5], [0, 1, 5, 4], [2, 3, 7, 6], [0, 1, 3, 2], [4, 5, 7, 6]]


def write_cell_dirs(root, cm: CellMeshes, one_based=True):
    """Elem_<c>/SubElem_0 (NVTR of cell c's fine mesh, cell-local ids) and its Face_id<f>.dat
    (the triangles of the cell's tets on box face f, Salome format, vertex ids = the cell's node
    ids + 1) for every cell."""
    for c in range(cm.n_cells):
        xyz, tets, mat, box = cm.cell(c)
        d = os.path.join(root, f"Elem_{c}", "SubElem_0")
        write_nvtr(d, xyz, tets, mat, one_based=one_based)
        for f in range(6):
            axis, side = f // 2, f % 2
            on = np.abs(xyz[:, axis] - box[2 * axis + side]) < 1e-12 * max(1.0, abs(box[2 * axis + side]))
            hit = on[tets]
            rows = np.nonzero(hit.sum(axis=1) == 3)[0]
            tris = np.array([tets[e][hit[e]] for e in rows], dtype=np.int64).reshape(-1, 3)
            nodes = np.unique(tris)
            loc = -np.ones(xyz.shape[0], np.int64)
            loc[nodes] = np.arange(nodes.size)
            write_salome_dat(os.path.join(d, f"Face_id{f}.dat"), xyz[nodes], loc[tris], vertex_ids=nodes + 1)


def write_macro_nvtr(directory, vertex_xyz, cell_vertex, mat=None):
    """The macro mesh as NVTR polyhedra: per cell `8 v0..v7 6 (4 face cycle)x6` (faces x0, x1,
    y0, y1, z0, z1), the polyhedral format MsFEM/MsFEM_Main.cpp:187 reads (k = -1), 0-based (the
    only form the reference reads correctly).  The face cycles hold the cell's LOCAL vertex
    numbers 0..7: the grid takes them as indices into the cell's own vertex list
    (geometry::Polyhedron::CreateSubMeshInSelf, Library/GeometryShape.h:2709-2733, and
    GetGlobalIdFace, :2783-2789); global ids there read past the list."""
    recs = []
    for cv in np.asarray(cell_vertex, dtype=np.int64):
        r = [8] + list(cv) + [6]
        for cyc in FACE_CYCLES:
            r += [4] + list(cyc)
        recs.append(np.array(r, dtype=np.int64))
    write_nvtr(directory, vertex_xyz, recs, mat, one_based=False)


def write_tecplot(path, xyz, tets, mat, values, names, zone="Elastic"):
    """The FEBLOCK tetrahedron file of FEM_Grid::printTecPlot3D (FEM/FEM_Grid.h:3367-3452): nodal
    x, y, z (%.10e), one CELLCENTERED block per value array (%.10lf), then the 1-based
    connectivity.  Elements of domain 10 (the reference's DEL_domain) leave the element count and
    the connectivity (their line stays, empty); the value blocks follow the reference's loop,
    which tests the domain of element `i` -- the value index -- for every element."""
    xyz = np.asarray(xyz, dtype=np.float64)
    tets = np.asarray(tets, dtype=np.int64)
    mat = np.asarray(mat)
    del_domain = 10
    lines = ['TITLE     = "numerical"\n', 'VARIABLES = "x"\n "y"\n "z"\n']
    lines += [f' "{n}"\n' for n in names]
    n_keep = int((mat != del_domain).sum())
    lines.append(f'ZONE T="{zone}"\n')
    lines.append(f" N={xyz.shape[0]},  E={n_keep}, F=FEBLOCK ET=Tetrahedron \n")
    lines.append(" VARLOCATION=(NODAL NODAL NODAL" + " CELLCENTERED" * len(values) + ")\n")
    for d in range(3):
        lines += [f"{v:.10e}\n" for v in xyz[:, d]]
        lines.append("\n")
    for i, val in enumerate(values):
        if mat[i] != del_domain:
            lines += [f"{v:.10f}\n" for v in np.asarray(val, dtype=np.float64)]
        lines.append("\n")
    for e in range(tets.shape[0]):
        if mat[e] != del_domain:
            lines.append("".join(f"{int(v) + 1} " for v in tets[e]))
        lines.append("\n")
    with open(path, "w") as f:
        f.write("".join(lines))


def elastic_result_fields(post):
    """The six cell fields the elasticity driver prints (FEM/FEM_Main.cpp:1042-1052) from
    System.postprocess_elastic's array: sigma_xx, sigma_yy, sigma_zz, VonMises_stress (the
    driver's own formulas), Uy, Uz."""
    names = ["sigma_xx", "sigma_yy", "sigma_zz", "VonMises_stress", "Uy", "Uz"]
    return [post[:, 19], post[:, 20], post[:, 21], post[:, 22], post[:, 1], post[:, 2]], names
