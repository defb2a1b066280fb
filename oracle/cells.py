"""Test infrastructure only: CPU restatement of the MsFEM Order1 cell-basis
construction (MsFEM/MsFEM_Grid.h:4795-5759, Grid_forMech_Poly_Order1::
CreateFunctionalSpaces) for one hexahedral macro cell with its own fine mesh.

The reference builds 8 vector basis functions per cell, one per macro vertex v:
  edges  (MsFEM_Grid.h:5061-5200): on each of the 12 cell edges a 1-D elasticity
         problem (FEM::FEM_1D_forElasticDeformation, FEM/FEM.h:3796) with the
         Point (1,1,1) at one end and 0 at the other, over the fine segments on
         the edge; each segment takes the material id of the first face triangle
         that holds it (:4900-4925), which is 0: the face triangles come from the
         cell's Salome face files, read without material ids;
  faces  (:5205-5340): on each of the 6 faces a 2-D elasticity problem
         (FEM_2D_forElasticDeformation, FEM/FEM.h:4367) over the fine triangles on
         the face, Dirichlet data on the face border from the two edge solutions
         that meet at v and 0 on the other two edges;
  volume (:5380-5510): the 3-D problem (FEM_3D_forElasticDeformation,
         FEM/FEM.h:2970) over the cell's tetrahedra with the face solutions of v
         on the three faces through v and 0 on the other three.
Every sub-problem uses the same element block (FEM/FEM_Grid.h:2147-2191 for
tetrahedra, :4429-4500 for triangles, :3649-3720 for segments):
  A[I][J][a][b] = |e| (lambda gJ_a gI_b + mu gI_a gJ_b + mu delta_ab gI.gJ),
with g the gradient of the P1 barycentric function inside the simplex's own
line / plane / volume and |e| its length / area / volume.

Here each sub-problem is assembled with scipy and solved exactly (sparse LU) on
the free nodes.  `order1_bases(..., solver=ref)` instead hands each
sub-problem to the reference's own driver (oracle/_ref), chaining them the way
MsFEM_Grid.h does.

Cell conventions shared with the GPU path: vertex b of the box
[x0,x1]x[y0,y1]x[z0,z1] sits at (x_{b&1}, y_{(b>>1)&1}, z_{(b>>2)&1}); face f
(0..5) is x=x0, x=x1, y=y0, y=y1, z=z0, z=z1.  Face and edge materials: order1_bases'
face_material="zero" (the default, as on the GPU) is the reference's construction (material 0 on
both; its face meshes come from Salome files without material ids) and equals the reference's own
bases (tests/test_msfem_reference.py); face_material="cells" gives a face triangle its
tetrahedron's material and an edge segment that of its triangle on the lower-numbered of the
edge's two faces.
"""
from __future__ import annotations

import numpy as np

FACE_AXIS = np.array([0, 0, 1, 1, 2, 2])
FACE_SIDE = np.array([0, 1, 0, 1, 0, 1])


def lame(E, nu):
    E = np.asarray(E, dtype=np.float64)
    nu = np.asarray(nu, dtype=np.float64)
    return E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))


def simplex_gradients(P):
    """P: [k+1, 3] vertices of a segment / triangle / tetrahedron -> (g [k+1, 3], measure)."""
    k = P.shape[0] - 1
    E = (P[1:] - P[0]).T                       # 3 x k edge vectors
    G = E.T @ E                                # k x k metric
    Ginv = np.linalg.inv(G)
    gk = (E @ Ginv).T                          # gradients of l_1..l_k inside the simplex's span
    g = np.vstack([-gk.sum(axis=0), gk])
    meas = np.sqrt(np.linalg.det(G)) / [1.0, 1.0, 2.0, 6.0][k]
    return g, meas


def element_block(g, meas, lam, mu):
    """[k+1, k+1, 3, 3] element blocks in the reference's orientation."""
    gg = g @ g.T
    A = lam * np.einsum("ja,ib->ijab", g, g) + mu * np.einsum("ia,jb->ijab", g, g)
    A += mu * gg[:, :, None, None] * np.eye(3)[None, None]
    return meas * A


def assemble(xyz, elems, mat, E, nu, textbook=False):
    """Global node-blocked matrix (DOF 3*node+c) as scipy CSR; the per-element formula of
    simplex_gradients / element_block, evaluated for all elements at once.  textbook=True:
    the textbook orientation K[I][J][a][b] = V (lambda gI_a gJ_b + mu gJ_a gI_b + ...), i.e. the
    reference's blocks transposed (symmetric positive semi-definite)."""
    import scipy.sparse as sp
    lam, mu = lame(E, nu)
    n = xyz.shape[0]
    elems = np.asarray(elems, dtype=np.int64)
    ne, k1 = elems.shape
    k = k1 - 1
    P = xyz[elems]                                  # [ne, k1, 3]
    Ed = P[:, 1:, :] - P[:, :1, :]                  # [ne, k, 3] edge vectors (rows)
    G = Ed @ Ed.transpose(0, 2, 1)                  # [ne, k, k]
    Ginv = np.linalg.inv(G)
    gk = Ginv @ Ed                                  # [ne, k, 3] gradients of l_1..l_k
    g = np.concatenate([-gk.sum(axis=1, keepdims=True), gk], axis=1)   # [ne, k1, 3]
    meas = np.sqrt(np.linalg.det(G)) / [1.0, 1.0, 2.0, 6.0][k]
    la, m_ = lam[mat][:, None, None, None, None], mu[mat][:, None, None, None, None]
    gg = np.einsum("eia,eja->eij", g, g)
    if textbook:
        A = la * np.einsum("eia,ejb->eijab", g, g) + m_ * np.einsum("eja,eib->eijab", g, g)
    else:
        A = la * np.einsum("eja,eib->eijab", g, g) + m_ * np.einsum("eia,ejb->eijab", g, g)
    A = A + (mu[mat][:, None, None] * gg)[:, :, :, None, None] * np.eye(3)[None, None, None]
    A *= meas[:, None, None, None, None]
    r = 3 * elems[:, :, None] + np.arange(3)[None, None, :]          # [ne, k1, 3] DOFs
    blk = A.transpose(0, 1, 3, 2, 4).reshape(ne, 3 * k1, 3 * k1)   # rows (I, a), cols (J, b)
    rr = r.reshape(ne, 3 * k1)
    rows = np.repeat(rr, 3 * k1, axis=1).ravel()
    cols = np.tile(rr, (1, 3 * k1)).ravel()
    return sp.csr_matrix((blk.ravel(), (rows, cols)), shape=(3 * n, 3 * n))


def residual(K, x, fixed_nodes):
    """Relative residual ||F_I - K_II x_I|| / ||F_I|| per right-hand side of x [n, R, 3]
    (F_I = -K_IB g), the measure the batched solver stops on."""
    n = x.shape[0]
    fixed = np.zeros(3 * n, bool)
    fixed[(3 * np.asarray(fixed_nodes)[:, None] + np.arange(3)).ravel()] = True
    out = []
    for r in range(x.shape[1]):
        xf = x[:, r, :].ravel()
        g = np.where(fixed, xf, 0.0)
        F = -(K @ g)[~fixed]
        res = F - K[~fixed][:, ~fixed] @ xf[~fixed]
        out.append(np.linalg.norm(res) / max(np.linalg.norm(F), 1e-300))
    return np.array(out)


def solve_dirichlet(K, n, bc_nodes, bc_values):
    """x with x[bc] = values and K_II x_I = -K_IB x_B (exact sparse LU)."""
    import scipy.sparse.linalg as spl
    x = np.zeros((n, 3))
    x[bc_nodes] = bc_values
    fixed = np.zeros(3 * n, bool)
    fixed[(3 * np.asarray(bc_nodes)[:, None] + np.arange(3)).ravel()] = True
    free = ~fixed
    xf = x.ravel()
    rhs = -(K[free][:, fixed] @ xf[fixed])
    if free.any():
        xf[free] = spl.spsolve(K[free][:, free].tocsc(), rhs)
    return xf.reshape(n, 3)


def cell_problem(dim, xyz, elems, mat, E, nu, bc_nodes, bc_values):
    K = assemble(xyz, elems, mat, E, nu)
    return solve_dirichlet(K, xyz.shape[0], bc_nodes, bc_values)


# --------------------------------------------------------------------------------------------
# Order1 orchestration for one cell
# --------------------------------------------------------------------------------------------

def face_masks(xyz, box, rel_tol=1e-9):
    """bit f set when the node lies on face f of the box [x0,x1,y0,y1,z0,z1]."""
    box = np.asarray(box, dtype=np.float64)
    size = max(box[1] - box[0], box[3] - box[2], box[5] - box[4])
    tol = rel_tol * size
    mask = np.zeros(xyz.shape[0], dtype=np.int32)
    for f in range(6):
        mask |= (np.abs(xyz[:, FACE_AXIS[f]] - box[f]) <= tol).astype(np.int32) << f
    return mask


def vertex_faces(v):
    """The three faces through vertex v."""
    return [0 + (v & 1), 2 + ((v >> 1) & 1), 4 + ((v >> 2) & 1)]


def cell_edges():
    """The 12 edges as (axis, face_a, face_b, v_low, v_high), face_a < face_b the two faces
    holding it, v_low / v_high the vertices at its low / high end along axis."""
    out = []
    for axis in range(3):
        others = [a for a in range(3) if a != axis]
        for s in range(2):
            for t in range(2):
                fa, fb = 2 * others[0] + s, 2 * others[1] + t
                bits = (s << others[0]) | (t << others[1])
                out.append((axis, fa, fb, bits, bits | (1 << axis)))
    return out


def face_triangles(tets, mat, mask):
    """Per face f: (triangles [t, 3] in tet-local node order, material [t]), tets in order."""
    out = []
    on = mask[tets]  # [E, 4]
    for f in range(6):
        hit = ((on >> f) & 1).astype(bool)
        rows = np.nonzero(hit.sum(axis=1) == 3)[0]
        tri = np.array([tets[e][hit[e]] for e in rows], dtype=np.int64).reshape(-1, 3)
        out.append((tri, mat[rows]))
    return out


def order1_bases(xyz, tets, mat, box, E, nu, solver=None, face_material="zero"):
    """Bases [n_nodes, 8, 3] of one Order1 cell.  solver(dim, xyz, elems, mat, E, nu, bc_nodes, bc_values)
    solves one sub-problem (default: the exact restatement `cell_problem`).  face_material:
    "zero" (default) -- material 0 everywhere, as the reference's construction has it (its face
    meshes come from Salome files, whose ReadFromSalomeDat leaves every material id 0,
    Library/Math.h:91-147, MsFEM_Grid.h:4848, and the edge segments copy the face ids, :4905);
    "cells" -- the face triangles and edge segments take the material of the tetrahedra they
    bound."""
    solve = solver or cell_problem
    xyz = np.asarray(xyz, dtype=np.float64)
    tets = np.asarray(tets, dtype=np.int64)
    mat = np.asarray(mat, dtype=np.int32)
    n = xyz.shape[0]
    mask = face_masks(xyz, box)
    vert = np.full(8, -1)
    for v in range(8):
        want = sum(1 << f for f in vertex_faces(v))
        hit = np.nonzero((mask & want) == want)[0]
        assert hit.size == 1, f"vertex {v}: {hit.size} nodes"
        vert[v] = hit[0]
    if face_material not in ("cells", "zero"):
        raise ValueError("face_material must be 'cells' or 'zero'")
    tris = face_triangles(tets, mat if face_material == "cells" else np.zeros_like(mat), mask)

    # edges: sorted nodes along the edge, segment materials, the two end profiles
    edge_sol = {}   # (edge id) -> (nodes [k], sol_low [k,3], sol_high [k,3])
    for ei, (axis, fa, fb, vl, vh) in enumerate(cell_edges()):
        want = (1 << fa) | (1 << fb)
        nodes = np.nonzero((mask & want) == want)[0]
        nodes = nodes[np.argsort(xyz[nodes, axis], kind="stable")]
        assert nodes[0] == vert[vl] and nodes[-1] == vert[vh]
        ftri, fmat = tris[fa]
        segs, smat = [], []
        for a, b in zip(nodes[:-1], nodes[1:]):
            has = np.nonzero(np.any(ftri == a, axis=1) & np.any(ftri == b, axis=1))[0]
            assert has.size >= 1, "edge segment without a face triangle"
            segs.append((a, b))
            smat.append(fmat[has[0]])
        loc = {int(g): i for i, g in enumerate(nodes)}
        el = np.array([[loc[a], loc[b]] for a, b in segs], dtype=np.int32)
        exyz = xyz[nodes]
        ends = np.array([0, nodes.size - 1], dtype=np.int32)
        s_lo = solve(1, exyz, el, np.array(smat, np.int32), E, nu, ends, np.array([[1.0, 1, 1], [0, 0, 0]]))
        s_hi = solve(1, exyz, el, np.array(smat, np.int32), E, nu, ends, np.array([[0.0, 0, 0], [1, 1, 1]]))
        edge_sol[ei] = (nodes, s_lo, s_hi)

    # faces: one problem per (face, vertex on the face)
    face_sol = {}   # (f, v) -> (nodes [k], sol [k,3])
    edges = cell_edges()
    for f in range(6):
        fnodes = np.nonzero((mask >> f) & 1)[0]
        loc = -np.ones(n, dtype=np.int64)
        loc[fnodes] = np.arange(fnodes.size)
        ftri, fmat = tris[f]
        border = np.nonzero(mask[fnodes] & ~(1 << f))[0]
        for v in range(8):
            if f not in vertex_faces(v):
                continue
            val = np.zeros((fnodes.size, 3))
            for ei, (axis, fa, fb, vl, vh) in enumerate(edges):
                if f not in (fa, fb) or v not in (vl, vh):
                    continue
                nodes, s_lo, s_hi = edge_sol[ei]
                val[loc[nodes]] = s_lo if v == vl else s_hi
            face_sol[(f, v)] = (fnodes, solve(2, xyz[fnodes], loc[ftri].astype(np.int32), fmat, E, nu,
                                              border.astype(np.int32), val[border]))

    # volume: one problem per vertex
    bnodes = np.nonzero(mask)[0].astype(np.int32)
    out = np.zeros((n, 8, 3))
    for v in range(8):
        val = np.zeros((n, 3))
        for f in sorted(vertex_faces(v), reverse=True):   # the lowest face through v is written last
            fnodes, s = face_sol[(f, v)]
            val[fnodes] = s
        out[:, v, :] = solve(3, xyz, tets.astype(np.int32), mat, E, nu, bnodes, val[bnodes])
    return out


# --------------------------------------------------------------------------------------------
# MsFEM macro element (FiniteElement_forMech_Poly_Order1::SolveLocalMatrix, MsFEM_Grid.h:3837-3975)
# --------------------------------------------------------------------------------------------

# vertex cycles of the six box faces (face order x0, x1, y0, y1, z0, z1)
FACE_CYCLES = np.array([[0, 2, 6, 4], [1, 3, 7, 5], [0, 1, 5, 4], [2, 3, 7, 6], [0, 1, 3, 2], [4, 5, 7, 6]])


def box_vertices(box):
    b = np.asarray(box, dtype=np.float64)
    return np.array([[b[0 + (v & 1)], b[2 + ((v >> 1) & 1)], b[4 + ((v >> 2) & 1)]] for v in range(8)])


def poly_quadrature(verts, faces=FACE_CYCLES):
    """Polyhedron::CreateSubMeshInSelf + SetIntegrationLaw(4) (Library/GeometryShape.h:2708-2760,
    :2820-2836): for each face, for each edge (v_i, v_i+1), the sub-tetrahedron (centroid, face
    centroid, v_i, v_i+1) with the 4-point rule u = (5 - sqrt 5)/20, weight V_sub / 4."""
    verts = np.asarray(verts, dtype=np.float64)
    C = verts.mean(axis=0)
    u = (5.0 - np.sqrt(5.0)) / 20.0
    v = 1.0 - 3.0 * u
    bary = np.array([[u, u, u], [v, u, u], [u, v, u], [u, u, v]])
    pts, w = [], []
    for f in faces:
        F = verts[f].mean(axis=0)
        for i in range(len(f)):
            P = np.array([C, F, verts[f[i]], verts[f[(i + 1) % len(f)]]])
            E = P[1:] - P[0]
            vol = abs(np.linalg.det(E)) / 6.0
            for b in bary:
                pts.append(P[0] + b @ E)
                w.append(vol / 4.0)
    return np.array(pts), np.array(w)


def isotropic_D(E, nu):
    """Domain::forMech isotropic D (Library/Domain.h:53-78): Voigt order xx, yy, zz, xy, yz, zx,
    engineering shear."""
    k = E * (1 - nu) / ((1 + nu) * (1 - 2 * nu))
    a = nu / (1 - nu)
    b = (1 - 2 * nu) / (2 * (1 - nu))
    D = np.zeros((6, 6))
    D[:3, :3] = k * a
    np.fill_diagonal(D[:3, :3], k)
    D[3, 3] = D[4, 4] = D[5, 5] = k * b
    return D


def locate(xyz, tets, x, tol=1e-12):
    """Index of the first tetrahedron containing x (barycentrics >= -tol), the micro element the
    reference's nearest-element lookup (GeometryGrid.h:323-340) returns for interior points."""
    P = xyz[tets]                                  # [E, 4, 3]
    E = P[:, 1:, :] - P[:, :1, :]                  # [E, 3, 3]
    lam = np.linalg.solve(np.transpose(E, (0, 2, 1)), (x - P[:, 0, :])[:, :, None])[:, :, 0]
    l0 = 1 - lam.sum(axis=1)
    inside = (lam.min(axis=1) >= -tol) & (l0 >= -tol)
    hit = np.nonzero(inside)[0]
    if hit.size == 0:
        raise ValueError("quadrature point outside the cell mesh")
    return int(hit[0])


def strain_matrix(G):
    """B (6 x 3) of the component-wise vector basis with gradient G[c][d] = d psi^c / dx_d, the rows
    of MsFEM_Grid.h:3868-3885 (column a: the strain of e_a psi^a)."""
    B = np.zeros((6, 3))
    B[0, 0], B[1, 1], B[2, 2] = G[0, 0], G[1, 1], G[2, 2]
    B[3, 0], B[3, 1] = G[0, 1], G[1, 0]
    B[4, 2], B[4, 1] = G[2, 1], G[1, 2]
    B[5, 2], B[5, 0] = G[2, 0], G[0, 2]
    return B


def macro_element_matrix(xyz, tets, bases, box, E0, nu0):
    """[8, 8, 3, 3]: A[I][J][r][c] = sum_q w_q (B_J^T D0 B_I)[r][c] over the macro quadrature, the
    basis gradients from the micro tetrahedron holding each point, D0 = domain 0's material
    (MsFEM/MsFEM.h:644-647)."""
    xyz = np.asarray(xyz, dtype=np.float64)
    tets = np.asarray(tets, dtype=np.int64)
    pts, w = poly_quadrature(box_vertices(box))
    D = isotropic_D(E0, nu0)
    A = np.zeros((8, 8, 3, 3))
    for x, wq in zip(pts, w):
        e = locate(xyz, tets, x)
        g, _ = simplex_gradients(xyz[tets[e]])              # [4, 3]
        Bs = []
        for I in range(8):
            G = bases[tets[e], I, :].T @ g                   # [3 comps, 3 derivs]
            Bs.append(strain_matrix(G))
        for I in range(8):
            DBI = D @ Bs[I]
            for J in range(8):
                A[I, J] += wq * (Bs[J].T @ DBI)
    return A
