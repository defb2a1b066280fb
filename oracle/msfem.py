"""Test infrastructure only: CPU restatement of the MsFEM Order1 elasticity driver
(MsFEM::MsFEM_forElasticDeformation_OrderBF1_forPoly, MsFEM/MsFEM.h:572-1010) on top of
oracle/cells.py: macro element matrices, macro boundary loads (BoundaryFace_forMech_Poly_Order1::
SolveLocalBoundaryVector, MsFEM_Grid.h:4104-4135 with the polygon rule of GeometryShape.h:
2563-2600 and the triangle 4-point rule of :1482-1540), assembly over the macro vertices, exact
Dirichlet elimination and a dense FP64 solve, and the fine solution on every cell."""
from __future__ import annotations

import numpy as np

from . import cells as oc


def polygon_quadrature(V4):
    """(points [16, 3], weights [16]) of geometry::Polygon with SetIntegrationLaw(4) over the
    vertex cycle V4 (GeometryShape.h:2563-2640): the fan of triangles (centroid, V_i, V_i+1), each
    with the 4-point rule of :1482-1540 (barycentric (1/3, 1/3), (3/5, 1/5), (1/5, 3/5), (1/5, 1/5)
    from the centroid; weights -9/32, 25/96 x3 times |e1 x e2|)."""
    V4 = np.asarray(V4, dtype=np.float64)
    F = V4.mean(axis=0)
    xs = [(1 / 3, 1 / 3, -9 / 32), (3 / 5, 1 / 5, 25 / 96), (1 / 5, 3 / 5, 25 / 96), (1 / 5, 1 / 5, 25 / 96)]
    pts, ws = [], []
    for i in range(4):
        e1, e2 = V4[i] - F, V4[(i + 1) % 4] - F
        detD = np.linalg.norm(np.cross(e1, e2))
        for x, y, w in xs:
            pts.append(F + e1 * x + e2 * y)
            ws.append(w * detD)
    return np.array(pts), np.array(ws)


def face_loads(xyz, tets, bases, box, face, traction):
    """[8, 3]: sum_q w_q t_a psi_v^a(x_q) over face `face` of the box (the component-wise
    product of SolveLocalBoundaryVector, MsFEM_Grid.h:4104-4135), psi interpolated linearly in the
    micro tetrahedron holding x_q."""
    pts, ws = polygon_quadrature(oc.box_vertices(box)[oc.FACE_CYCLES[face]])
    out = np.zeros((8, 3))
    for p, w in zip(pts, ws):
        e = oc.locate(xyz, tets, p)
        P = xyz[tets[e]]
        lam = np.linalg.solve((P[1:] - P[0]).T, p - P[0])
        lam = np.concatenate([[1 - lam.sum()], lam])
        psi = np.einsum("k,kva->va", lam, bases[tets[e]])
        out += w * np.asarray(traction)[None, :] * psi
    return out


def driver(cc, bases, fixed_vertices, fixed_values, items, tractions, E0, nu0):
    """(U [n_vertices, 3], u_cells [cell nodes, 3], K, F) with the given cell bases."""
    cm = cc.cells
    nv = cc.n_coarse_vertices
    A = np.zeros((3 * nv, 3 * nv))
    Ks = []
    for c in range(cm.n_cells):
        xyz, tets, mat, box = cm.cell(c)
        B = bases[cm.node_off[c]:cm.node_off[c + 1]]
        K = oc.macro_element_matrix(xyz, tets, B, box, E0, nu0)
        Ks.append(K)
        for I in range(8):
            for J in range(8):
                vi, vj = cc.cell_vertex[c, I], cc.cell_vertex[c, J]
                A[3 * vi:3 * vi + 3, 3 * vj:3 * vj + 3] += K[I, J]
    F = np.zeros((nv, 3))
    for (c, f), t in zip(items, tractions):
        xyz, tets, mat, box = cm.cell(c)
        F[cc.cell_vertex[c]] += face_loads(xyz, tets, bases[cm.node_off[c]:cm.node_off[c + 1]], box, f, t)
    x = np.zeros(3 * nv)
    fixed = np.zeros(3 * nv, bool)
    for v, val in zip(fixed_vertices, fixed_values):
        fixed[3 * v:3 * v + 3] = True
        x[3 * v:3 * v + 3] = val
    free = ~fixed
    rhs = F.ravel()[free] - A[free][:, fixed] @ x[fixed]
    x[free] = np.linalg.solve(A[free][:, free], rhs)
    U = x.reshape(nv, 3)
    u = np.zeros((cm.xyz.shape[0], 3))
    for c in range(cm.n_cells):
        a, b = cm.node_off[c], cm.node_off[c + 1]
        u[a:b] = np.einsum("vk,nvk->nk", U[cc.cell_vertex[c]], bases[a:b])
    return U, u, np.array(Ks), F
