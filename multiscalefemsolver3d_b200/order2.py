"""MsFEM Order2 (MsFEM/MsFEM.h:14-569, MsFEM_Grid.h:1001-3470) on the GPU: the macro topology and
DOF numbering of a box macro mesh and the Dirichlet groups' DOF and face lists on the host; the
cells' 27 bases (msfem_cells_build_order2) and the macro phase (msfem_cells_order2_macro_solve:
element matrices, the macro system, the Dirichlet values as the L2 projection Grid_forMech::
CreateBoundaryConditions makes, :3303-3470, their elimination and the solve) on the device.

Macro mesh conventions: cell c's corners cell_vertex[c][b] sit at the box vertex b
(x_{b&1}, y_{(b>>1)&1}, z_{(b>>2)&1}); its faces are the cycles FACE_CYCLES (x0, x1, y0, y1,
z0, z1) as meshio.write_macro_nvtr writes them.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import FP32_IR, check, load

__all__ = ["FACE_CYCLES", "MacroTopology", "macro_topology", "DirichletLayout", "dirichlet_layout", "macro_system",
           "dirichlet_projection", "order2_elastic_driver"]

FACE_CYCLES = np.array([[0, 2, 6, 4], [1, 3, 7, 5], [0, 1, 5, 4], [2, 3, 7, 6], [0, 1, 3, 2], [4, 5, 7, 6]])


@dataclass
class MacroTopology:
    edges: np.ndarray        # [NE, 2] (lower, higher) vertex ids, ascending
    faces: np.ndarray        # [NF, 4] vertex cycles, ascending lexicographically
    face_edges: np.ndarray   # [NF, 4] the edge between cycle nodes k and k+1
    cell_faces: np.ndarray   # [nc, 6]
    cell_dofs: np.ndarray    # [nc, 27]
    n_vertices: int

    @property
    def n_dofs(self) -> int:
        return self.n_vertices + len(self.edges) + len(self.faces) + len(self.cell_faces)


def macro_topology(cell_vertex, n_vertices=None) -> MacroTopology:
    """The reference's CreateTopology (MsFEM_Grid.h:427-997) for box cells: faces are the distinct
    global vertex cycles in lexicographic order, edges the distinct (lower, higher) pairs in order;
    a cell's 27 DOFs are its vertices, NV + its edges (ascending), NV + NE + its faces (local
    order), NV + NE + NF + the cell (:3045-3054)."""
    cv = np.asarray(cell_vertex, dtype=np.int64)
    nc = cv.shape[0]
    nv = int(cv.max()) + 1 if n_vertices is None else int(n_vertices)
    cyc = cv[:, FACE_CYCLES].reshape(-1, 4)                              # [6 nc, 4]
    faces, finv = np.unique(cyc, axis=0, return_inverse=True)
    a, b = faces, np.roll(faces, -1, axis=1)
    pairs = np.stack([np.minimum(a, b), np.maximum(a, b)], axis=2).reshape(-1, 2)
    edges, einv = np.unique(pairs, axis=0, return_inverse=True)
    face_edges = einv.reshape(-1, 4)
    cell_faces = finv.reshape(nc, 6)
    ne, nf = len(edges), len(faces)
    ce = np.sort(face_edges[cell_faces].reshape(nc, 24), axis=1)
    cell_edges = np.array([np.unique(r) for r in ce])                   # 12 per box cell
    if cell_edges.shape != (nc, 12):
        raise ValueError("cells are not boxes with 12 distinct edges")
    dofs = np.concatenate([cv, nv + cell_edges, nv + ne + cell_faces, (nv + ne + nf + np.arange(nc))[:, None]], axis=1)
    return MacroTopology(edges, faces, face_edges, cell_faces, dofs.astype(np.int64), nv)


@dataclass
class DirichletLayout:
    """The integer bookkeeping of the Order2 Dirichlet groups, as msfem_cells_order2_dirichlet and
    msfem_cells_order2_macro_solve take it."""
    faces: np.ndarray           # int32 [n_faces, 10]: cell, 9 DOF ids (4 cycle vertices, 4 edges, face)
    group_dof_off: np.ndarray   # int32 [n_groups + 1]
    group_dofs: np.ndarray      # int32: each group's DOFs, ascending
    group_face_off: np.ndarray  # int32 [n_groups + 1]
    group_values: np.ndarray    # float64 [n_groups, 3]
    fixed_dofs: np.ndarray      # int32: scalar rows 3 d + c in elimination order
    fixed_src: np.ndarray       # int32: 3 k + c into the projected values [group DOF k][c]


def dirichlet_layout(topo: MacroTopology, groups) -> DirichletLayout:
    """Per Dirichlet group (vertex ids, value (3,), take (3 bools)) -- Grid_forMech::
    CreateBoundaryConditions, MsFEM_Grid.h:3303-3470 -- its DOFs (the vertices, the edges with both
    ends in it, the faces with all four vertices in it, ascending), its faces (ascending face id,
    each on one cell only) with their 9 DOFs (the cycle vertices, the edges between cycle nodes k
    and k + 1, the face), and the rows to eliminate: each group DOF in order, each taken component
    (scalar row 3 d + c).  A row named twice is eliminated once, at its first place, with the
    later group's value (the reference would already have moved the earlier value into the other
    rows by then, MsFEM.h:300-365; that inconsistency is not copied)."""
    nv, ne, nf = topo.n_vertices, len(topo.edges), len(topo.faces)
    nc = topo.cell_faces.shape[0]
    count = np.bincount(topo.cell_faces.ravel(), minlength=nf)
    face_cell = np.full(nf, -1, np.int64)
    face_cell[topo.cell_faces.ravel()] = np.repeat(np.arange(nc), 6)
    faces, dof_off, dofs, face_off, values = [], [0], [], [0], []
    rows, src = [], []
    for verts, value, take in groups:
        verts = np.unique(np.asarray(verts, dtype=np.int64))
        inside = np.zeros(nv, bool)
        inside[verts] = True
        on_e = np.nonzero(inside[topo.edges[:, 0]] & inside[topo.edges[:, 1]])[0]
        tf = np.nonzero(inside[topo.faces].all(axis=1))[0]
        gd = np.sort(np.concatenate([verts, nv + on_e, nv + ne + tf]))
        for f in tf:
            if count[f] != 1:
                raise ValueError(f"Dirichlet face {f} is shared by two cells")
            faces.append(np.concatenate([[face_cell[f]], topo.faces[f], nv + topo.face_edges[f], [nv + ne + f]]))
        base = dof_off[-1]
        for k, d in enumerate(gd):
            for comp in range(3):
                if take[comp]:
                    rows.append(3 * int(d) + comp)
                    src.append(3 * (base + k) + comp)
        dofs.append(gd)
        dof_off.append(base + len(gd))
        face_off.append(face_off[-1] + len(tf))
        values.append(np.asarray(value, dtype=np.float64).reshape(3))
    last = {}
    for r, i in zip(rows, src):
        last[r] = i
    return DirichletLayout(
        faces=np.asarray(faces, np.int32).reshape(-1, 10),
        group_dof_off=np.asarray(dof_off, np.int32),
        group_dofs=(np.concatenate(dofs) if dofs else np.zeros(0)).astype(np.int32),
        group_face_off=np.asarray(face_off, np.int32),
        group_values=np.asarray(values, np.float64).reshape(-1, 3),
        fixed_dofs=np.asarray(list(last.keys()), np.int32),
        fixed_src=np.asarray(list(last.values()), np.int32))


def _args(topo: MacroTopology, vertex_xyz, lay: DirichletLayout):
    P = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    keep = [np.ascontiguousarray(topo.cell_dofs, dtype=np.int32), np.ascontiguousarray(vertex_xyz, dtype=np.float64)]
    keep += [np.ascontiguousarray(a) for a in (lay.faces, lay.group_dof_off, lay.group_dofs, lay.group_face_off,
                                               lay.group_values)]
    cd, vx, fa, do, gd, fo, gv = keep
    args = [topo.n_dofs, P(cd), vx.shape[0], P(vx), fa.shape[0], P(fa), gv.shape[0], P(do), P(gd), P(fo), P(gv)]
    return args, keep


def macro_system(cells_gpu, topo: MacroTopology):
    """The Order2 macro system on the device (msfem_cells_order2_macro_system): a matrix-only
    fem.System, scalar rows 3 d + c, from the built Order2 bases of `cells_gpu` (cells.Cells)."""
    from .fem import System
    cd = np.ascontiguousarray(topo.cell_dofs, dtype=np.int32)
    h = C.c_void_p()
    check(load().msfem_cells_order2_macro_system(cells_gpu.h, topo.n_dofs, cd.ctypes.data_as(C.c_void_p),
                                                 C.byref(h)), "cells_order2_macro_system")
    return System._from_handle(h)


def dirichlet_projection(cells_gpu, topo: MacroTopology, vertex_xyz, lay: DirichletLayout):
    """The projected Dirichlet values [len(lay.group_dofs), 3] on the device
    (msfem_cells_order2_dirichlet)."""
    args, keep = _args(topo, vertex_xyz, lay)
    out = np.empty((max(1, lay.group_dofs.size), 3))
    check(load().msfem_cells_order2_dirichlet(cells_gpu.h, *args, out.ctypes.data_as(C.c_void_p)),
          "cells_order2_dirichlet")
    return out[:lay.group_dofs.size]


def order2_elastic_driver(cells, vertex_xyz, cell_vertex, groups, precision=FP32_IR, tol=1e-8, cell_tol=1e-8,
                          maxiter=200000):
    """MsFEM_forElasticDeformation_OrderBF2_forPoly on the GPU: returns (macro solution [n_dofs, 3],
    info).  The cell bases (msfem_cells_build_order2) and the whole macro phase
    (msfem_cells_order2_macro_solve: element matrices, the macro system, the projected Dirichlet
    values, their elimination by rows and columns, MINRES with FP32 inner solves in FP64
    refinement by default, to ||F - A x|| <= tol ||F||) run on the device; the host computes the
    macro topology and the groups' DOF and face lists.  The reference runs plain CG restarts on
    the same system (MsFEM.h:445-478)."""
    from .cells import Cells
    vertex_xyz = np.asarray(vertex_xyz, dtype=np.float64)
    topo = macro_topology(cell_vertex, n_vertices=vertex_xyz.shape[0])
    lay = dirichlet_layout(topo, groups)
    args, keep = _args(topo, vertex_xyz, lay)
    fd = np.ascontiguousarray(lay.fixed_dofs, dtype=np.int32)
    fs = np.ascontiguousarray(lay.fixed_src, dtype=np.int32)
    U = np.empty((topo.n_dofs, 3))
    it, rel = C.c_int32(), C.c_double()
    P = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    cg = Cells(cells)
    try:
        cg.build_order2(np.asarray(cell_vertex, np.int32), precision, cell_tol)
        rc = check(load().msfem_cells_order2_macro_solve(cg.h, *args, fd.size, P(fd), P(fs), precision, tol, maxiter,
                                                         P(U), C.byref(it), C.byref(rel)), "cells_order2_macro_solve")
    finally:
        cg.close()
    return U, {"rel_residual": rel.value, "iterations": it.value, "rc": rc, "n_dofs": topo.n_dofs}
