"""Test infrastructure only: CPU restatement of the MsFEM Order2 cell-basis construction
(MsFEM/MsFEM_Grid.h:1001-3080, Grid_forMech::CreateFunctionalSpaces) for one hexahedral macro
cell of a box macro mesh, and of the Order2 macro element matrix (FiniteElement_forMech_Poly::
SolveLocalMatrix, :34-171).

The reference builds 27 vector basis functions per cell, numbered vertex -> edge -> face -> cell
(:3045-3054): the 8 cell vertices in the element's own vertex order, the 12 cell edges in
ascending global edge id, the 6 faces in the element's local face order, then the cell bubble.
Each is the solution of one fine 3-D elasticity problem (FEM_3D_forElasticDeformation,
FEM/FEM.h:2970) whose Dirichlet data on the cell faces chains face problems (FEM_2D, :4367),
which chain edge problems (FEM_1D, :3796):

  edges (:1197-1425), per cell edge, over its fine segments:
      two linear problems, (1,1,1) at one end and 0 at the other, and a bubble problem with
      zero ends and the source -[(l+m) H 1 + m tr(H) 1] of phi = 4 xi (1 - xi) along the edge
      (H = -8 / L^2 t t^T, t the edge's unit direction);
  faces (:1426-2180), per cell face, over its fine triangles:
      4 linear problems (the face vertex v: the edge-linear solutions that are 1 at v on the two
      face edges through v, 0 on the other two), 4 edge-bubble problems (the edge's bubble
      solution on that edge, 0 elsewhere) and 1 face-bubble problem (0 on the border).  The
      reference writes a source for the bubble problems (:1686-1731, :1975-2010), but
      FEM_2D_forElasticDeformation adds its element loads to the system only when it prints its
      log (FEM/FEM.h:4479-4490, `if (is_print_logFile) for (...) SummPartOfVector`), and the
      cell construction calls it with false: the face problems have no source, so the face
      edge bubbles are the elastic extensions of the edge bubbles and the face bubble is 0;
  volume (:2181-2920), over the cell's tetrahedra:
      8 linear problems (the face-linear solutions of v on the faces through v, 0 elsewhere,
      no source), 12 edge-bubble problems (the two faces' edge-bubble solutions, source of
      b(xi_x) times the two linear functions that are 1 on the edge, frame (edge, centroid of the
      last local face holding it)), 6 face-bubble problems (the face-bubble solution on the
      face, source of b(xi_x) b(xi_y) times the linear function that is 1 on the face, frame
      (face's first edge, face centroid)), 1 cell bubble (0 on every face, source of
      b(xi_x) b(xi_y) b(xi_z) in the global frame, xi over the cell's bounding box).

Every source is the operator applied to its phi the way the reference writes it: with H the
Hessian of phi in global coordinates (H = A^T H_self A, A the frame's rows),
  f = -[(lambda + mu) H (1,1,1) + mu tr(H) (1,1,1)],
lambda and mu of the fine element's material.  The sub-problem loads are the integrals of
f . phi_I with each element's own 4-point rule (segments: Gauss-Legendre, GeometryShape.h:746-925;
tetrahedra: :1754-1851), FEM/FEM_Grid.h:2521-2566, :3738-3783.

Every sub-problem here is solved exactly.  The reference solves each with a tolerance-escalation
restart loop (FEM/FEM.h:3704-3771 and alike) that returns its previous best iterate when a pass
meets MIN_RESIDUAL = 1e-15 -- on an edge of few or uniform segments the first pass does, and the
edge solution comes back as its initial guess (0 inside).  That loss is not reproduced.

The edge and face problems read their meshes from the cell's Face_id<f>.dat files, whose
ReadFromSalomeDat (Library/Math.h:91-147) leaves every material id 0: the edge and face problems
use domain 0's material whatever the tetrahedra next to them are made of.

The macro basis functions replicate each fine basis's z component into x and y (:2978-2979), so
the macro element matrix is the Order1 one (polyhedron quadrature, nearest micro element,
D of domain 0) over 27 such bases.
"""
from __future__ import annotations

import os

import numpy as np

from . import cells as oc

# faces of a box cell as vertex cycles (x0, x1, y0, y1, z0, z1), the macro-mesh writer's order
FACE_CYCLES = np.array([[0, 2, 6, 4], [1, 3, 7, 5], [0, 1, 5, 4], [2, 3, 7, 6], [0, 1, 3, 2], [4, 5, 7, 6]])

_GL4_X = np.array([np.sqrt((3 - 2 * np.sqrt(6 / 5)) / 7), np.sqrt((3 + 2 * np.sqrt(6 / 5)) / 7)])
_GL4 = (np.array([_GL4_X[0], _GL4_X[1], -_GL4_X[1], -_GL4_X[0]]),
        np.array([(18 + np.sqrt(30)) / 36, (18 - np.sqrt(30)) / 36, (18 - np.sqrt(30)) / 36, (18 + np.sqrt(30)) / 36]))


def _rule(dim):
    """(barycentric coordinates [q, dim+1], weights [q] relative to the element measure)."""
    if dim == 1:
        s = (1 + _GL4[0]) / 2
        return np.stack([1 - s, s], axis=1), _GL4[1] / 2
    u = (5 - np.sqrt(5)) / 20
    v = 1 - 3 * u
    b = np.array([[u, u, u], [v, u, u], [u, v, u], [u, u, v]])
    return np.column_stack([1 - b.sum(1), b]), np.full(4, 0.25)


def load_vector(xyz, elems, source):
    """F [n, 3]: sum over elements of the rule's points of w |e| f(x) phi_I(x); source(e_idx,
    points [ne, q, 3]) -> [ne, q, 3]."""
    elems = np.asarray(elems, dtype=np.int64)
    dim = elems.shape[1] - 1
    bary, w = _rule(dim)
    P = xyz[elems]                                               # [ne, k1, 3]
    _, meas = _measures(P)
    pts = np.einsum("qi,eic->eqc", bary, P)                      # [ne, q, 3]
    f = source(np.arange(elems.shape[0]), pts)                   # [ne, q, 3]
    contrib = np.einsum("q,e,eqc,qi->eic", w, meas, f, bary)     # [ne, k1, 3]
    F = np.zeros((xyz.shape[0], 3))
    np.add.at(F, elems, contrib)
    return F


def _measures(P):
    Ed = P[:, 1:, :] - P[:, :1, :]
    G = Ed @ Ed.transpose(0, 2, 1)
    k = P.shape[1] - 1
    return G, np.sqrt(np.linalg.det(G)) / [1.0, 1.0, 2.0, 6.0][k]


def solve(dim, xyz, elems, mat, E, nu, bc_nodes, bc_values, F=None):
    """The sub-problem with Dirichlet data (all three components) and load F, solved exactly."""
    import scipy.sparse.linalg as spl
    K = oc.assemble(xyz, elems, mat, E, nu)
    n = xyz.shape[0]
    x = np.zeros((n, 3))
    x[bc_nodes] = bc_values
    fixed = np.zeros(3 * n, bool)
    fixed[(3 * np.asarray(bc_nodes)[:, None] + np.arange(3)).ravel()] = True
    free = ~fixed
    xf = x.ravel()
    rhs = -(K[free][:, fixed] @ xf[fixed])
    if F is not None:
        rhs = rhs + F.ravel()[free]
    if free.any():
        xf[free] = spl.spsolve(K[free][:, free].tocsc(), rhs)
    return xf.reshape(n, 3)


def operator_source(H, lam, mu):
    """-[(lambda + mu) H 1 + mu tr(H) 1] for Hessians H [..., 3, 3] and Lame [...]."""
    d = H.sum(axis=-1)
    tr = np.trace(H, axis1=-2, axis2=-1)
    return -((lam + mu)[..., None] * d + (mu * tr)[..., None])


def triangle_frame(p0, p1, p2):
    """Rows X, Y, Z of an orthonormal frame of the triangle (p0, p1, p2): X along p1 - p0, Y in its
    plane, Z normal (geometry::Triangle::CreateSelfBasis, GeometryShape.h:978-1125).  Every source
    that uses the frame is unchanged when Y or Z changes sign, so only X's direction matters."""
    X = p1 - p0
    X = X / np.linalg.norm(X)
    n = np.cross(p1 - p0, p2 - p0)
    Z = n / np.linalg.norm(n)
    Y = np.cross(Z, X)
    return np.array([X, Y, Z])


def _bub(s):
    return -4 * s * s + 4 * s


def _dbub(s, h):
    return -8 / h * s + 4 / h


def _is_equal(a, b):
    """math::IsEqual (Library/Math.h): |a - b| < 1e-10."""
    return abs(a - b) < 1e-10


class _Topo:
    """The reference's topology of one box cell in a macro mesh: global ids of its 8 vertices ->
    its edges (lower id first, as CreateTopology stores them, MsFEM_Grid.h:597-612, :746-760) in
    ascending global id (= ascending (min, max) vertex pair), and each face's first edge."""

    def __init__(self, gvert):
        self.gvert = np.asarray(gvert, dtype=np.int64)
        pairs = set()
        for cyc in FACE_CYCLES:
            for k in range(4):
                a, b = cyc[k], cyc[(k + 1) % 4]
                ga, gb = self.gvert[a], self.gvert[b]
                pairs.add((a, b) if ga < gb else (b, a))
        # local (low, high) vertex pairs, ordered by their global (min, max) ids
        self.edges = sorted(pairs, key=lambda p: (self.gvert[p[0]], self.gvert[p[1]]))
        self.face_edges = []      # per face: its 4 edges (indices into self.edges) in cycle order
        for cyc in FACE_CYCLES:
            fe = []
            for k in range(4):
                a, b = cyc[k], cyc[(k + 1) % 4]
                fe.append(self.edge_index(a, b))
            self.face_edges.append(fe)

    def edge_index(self, a, b):
        key = (a, b) if self.gvert[a] < self.gvert[b] else (b, a)
        return self.edges.index(key)


def order2_bases(xyz, tets, mat, box, E, nu, gvert, parts=None):
    """Bases [n_nodes, 27, 3] of one Order2 cell (module docstring).  gvert: the global ids of the
    cell's 8 vertices (they fix the edge order and orientation)."""
    xyz = np.asarray(xyz, dtype=np.float64)
    tets = np.asarray(tets, dtype=np.int64)
    mat = np.asarray(mat, dtype=np.int32)
    E = np.asarray(E, dtype=np.float64)
    nu = np.asarray(nu, dtype=np.float64)
    lam, mu = oc.lame(E, nu)
    n = xyz.shape[0]
    topo = _Topo(gvert)
    V = oc.box_vertices(box)
    mask = oc.face_masks(xyz, box)
    vert = np.full(8, -1)
    for v in range(8):
        want = sum(1 << f for f in oc.vertex_faces(v))
        hit = np.nonzero((mask & want) == want)[0]
        assert hit.size == 1
        vert[v] = hit[0]
    tris = oc.face_triangles(tets, mat, mask)
    face_of = [set(c.tolist()) for c in FACE_CYCLES]

    # ---- edges: nodes along the edge, 2 linear + 1 bubble solutions
    edge_nodes, edge_sol = [], []
    for (a, b) in topo.edges:
        fa = [f for f in range(6) if a in face_of[f] and b in face_of[f]]
        want = (1 << fa[0]) | (1 << fa[1])
        nodes = np.nonzero((mask & want) == want)[0]                # ascending cell node id
        ftri = tris[fa[0]][0]
        segs = []
        for e in range(ftri.shape[0]):
            on = [v for v in ftri[e] if (mask[v] & want) == want]
            if len(on) == 2:
                segs.append(on)
        loc = {int(g): i for i, g in enumerate(nodes)}
        el = np.array([[loc[p], loc[q]] for p, q in segs], dtype=np.int32)
        exyz = xyz[nodes]
        smat = np.zeros(el.shape[0], np.int32)                       # Salome faces: material 0
        ends = np.array([loc[vert[a]], loc[vert[b]]])
        s_a = solve(1, exyz, el, smat, E, nu, ends, np.array([[1.0, 1, 1], [0, 0, 0]]))
        s_b = solve(1, exyz, el, smat, E, nu, ends, np.array([[0.0, 0, 0], [1, 1, 1]]))
        t = V[b] - V[a]
        L = np.linalg.norm(t)
        t = t / L
        Hs = (-8 / L ** 2) * np.outer(t, t)
        f0 = operator_source(Hs[None], lam[:1], mu[:1])[0]           # domain 0, constant
        F = load_vector(exyz, el, lambda e, p: np.broadcast_to(f0, p.shape))
        s_bub = solve(1, exyz, el, smat, E, nu, ends, np.zeros((2, 3)), F)
        edge_nodes.append(nodes)
        edge_sol.append({a: s_a, b: s_b, "bubble": s_bub})

    # ---- faces
    face_nodes, face_lin, face_ebub, face_bub = [], [], [], []
    for f in range(6):
        fn = np.nonzero((mask >> f) & 1)[0]
        loc = -np.ones(n, dtype=np.int64)
        loc[fn] = np.arange(fn.size)
        ftri = loc[tris[f][0]].astype(np.int32)
        fmat = np.zeros(ftri.shape[0], np.int32)
        fxyz = xyz[fn]
        border = np.nonzero(mask[fn] & ~(1 << f))[0]
        cyc = FACE_CYCLES[f]
        lin = {}
        for k in range(4):
            v = cyc[k]
            val = np.zeros((fn.size, 3))
            for ei in topo.face_edges[f]:
                if v in topo.edges[ei]:
                    val[loc[edge_nodes[ei]]] = edge_sol[ei][v]
            lin[v] = solve(2, fxyz, ftri, fmat, E, nu, border, val[border])
        ebub = {}
        for ei in topo.face_edges[f]:
            a, b = topo.edges[ei]
            val = np.zeros((fn.size, 3))
            val[loc[edge_nodes[ei]]] = edge_sol[ei]["bubble"]
            ebub[ei] = solve(2, fxyz, ftri, fmat, E, nu, border, val[border])
        bub = np.zeros((fn.size, 3))
        face_nodes.append(fn)
        face_lin.append(lin)
        face_ebub.append(ebub)
        face_bub.append(bub)

    if parts is not None:
        parts.update(edge_nodes=edge_nodes, edge_sol=edge_sol, face_nodes=face_nodes, face_lin=face_lin,
                     face_ebub=face_ebub, face_bub=face_bub, topo=topo)

    # ---- volume
    bnodes = np.nonzero(mask)[0].astype(np.int32)
    out = np.zeros((n, 27, 3))

    def vol_solve(vals_by_face, F=None):
        val = np.zeros((n, 3))
        for f in sorted(vals_by_face, reverse=True):    # the lowest face is written last
            val[face_nodes[f]] = vals_by_face[f]
        return solve(3, xyz, tets, mat, E, nu, bnodes, val[bnodes], F)

    for v in range(8):
        out[:, v] = vol_solve({f: face_lin[f][v] for f in range(6) if v in face_of[f]})
    for i, (a, b) in enumerate(topo.edges):
        fs = [f for f in range(6) if a in face_of[f] and b in face_of[f]]
        base = fs[-1]
        A = triangle_frame(V[a], V[b], V[FACE_CYCLES[base]].mean(axis=0))
        src = _volume_source(A, V, V[a], "edge")
        F = load_vector(xyz, tets, lambda e, p: src(p, lam[mat[e]], mu[mat[e]]))
        out[:, 8 + i] = vol_solve({f: face_ebub[f][topo.edge_index(a, b)] for f in fs}, F)
    for f in range(6):
        a, b = topo.edges[topo.face_edges[f][0]]
        A = triangle_frame(V[a], V[b], V[FACE_CYCLES[f]].mean(axis=0))
        src = _volume_source(A, V, V[a], "face")
        F = load_vector(xyz, tets, lambda e, p: src(p, lam[mat[e]], mu[mat[e]]))
        out[:, 20 + f] = vol_solve({f: face_bub[f]}, F)
    src = _volume_source(np.eye(3), V, V[0], "cell")
    F = load_vector(xyz, tets, lambda e, p: src(p, lam[mat[e]], mu[mat[e]]))
    out[:, 26] = vol_solve({}, F)
    return out


def _volume_source(A, V, e0, kind):
    """MsFEM_Grid.h:2371-2480 (edge bubbles), :2598-2700 (face bubbles), :2770-2830 (cell
    bubble): phi a product of per-axis factors over the cell's bounding box in the frame A."""
    s = V @ A.T
    down, up = s.min(axis=0), s.max(axis=0)
    h = up - down
    es = A @ e0

    def lin(axis):
        # (phi, dphi, d2phi) factor that is 1 on the side of the edge / face, 0 on the other
        if _is_equal(es[axis], down[axis]):
            return (lambda k: 1 - k), -1 / h[axis]
        return (lambda k: k), 1 / h[axis]

    def f(p, lam, mu):
        q = p @ A.T
        k = (q - down) / h
        fac = []
        for ax in range(3):
            quad = (kind == "cell") or (ax == 0) or (ax == 1 and kind == "face")
            if quad:
                fac.append((_bub(k[..., ax]), _dbub(k[..., ax], h[ax]), np.full(k.shape[:-1], -8 / h[ax] ** 2)))
            else:
                phi, d = lin(ax)
                fac.append((phi(k[..., ax]), np.full(k.shape[:-1], d), np.zeros(k.shape[:-1])))
        (px, dx, ddx), (py, dy, ddy), (pz, dz, ddz) = fac
        Hs = np.zeros(k.shape[:-1] + (3, 3))
        Hs[..., 0, 0] = ddx * py * pz
        Hs[..., 1, 1] = px * ddy * pz
        Hs[..., 2, 2] = px * py * ddz
        Hs[..., 0, 1] = Hs[..., 1, 0] = dx * dy * pz
        Hs[..., 0, 2] = Hs[..., 2, 0] = dx * py * dz
        Hs[..., 1, 2] = Hs[..., 2, 1] = px * dy * dz
        H = np.einsum("ai,...ab,bj->...ij", A, Hs, A)
        lam_b = np.broadcast_to(np.asarray(lam)[:, None], k.shape[:-1])
        mu_b = np.broadcast_to(np.asarray(mu)[:, None], k.shape[:-1])
        return operator_source(H, lam_b, mu_b)
    return f


def macro_element_matrix(xyz, tets, bases, box, E0, nu0):
    """[27, 27, 3, 3] Order2 macro element matrix: the Order1 quadrature and lookup over the 27
    bases with their z component in all three components (MsFEM_Grid.h:2941-2979)."""
    b = np.repeat(np.asarray(bases)[:, :, 2:3], 3, axis=2)
    return _macro(xyz, tets, b, box, E0, nu0)


def _macro(xyz, tets, bases, box, E0, nu0):
    xyz = np.asarray(xyz, dtype=np.float64)
    tets = np.asarray(tets, dtype=np.int64)
    nb = bases.shape[1]
    pts, w = oc.poly_quadrature(oc.box_vertices(box))
    D = oc.isotropic_D(E0, nu0)
    A = np.zeros((nb, nb, 3, 3))
    for x, wq in zip(pts, w):
        e = oc.locate(xyz, tets, x)
        g, _ = oc.simplex_gradients(xyz[tets[e]])
        Bs = [oc.strain_matrix(bases[tets[e], I, :].T @ g) for I in range(nb)]
        for I in range(nb):
            DBI = D @ Bs[I]
            for J in range(nb):
                A[I, J] += wq * (Bs[J].T @ DBI)
    return A


# --------------------------------------------------------------------------------------------
# Macro topology and the reference's own Order2 construction (oracle/_ref/order2_ref)
# --------------------------------------------------------------------------------------------

def macro_topology(cell_vertex):
    """The reference's CreateTopology (MsFEM_Grid.h:427-997) on box cells written with FACE_CYCLES:
    faces = distinct global vertex cycles in ascending lexicographic order, edges = distinct
    (lower, higher) vertex pairs in ascending order, each face's edges in cycle order.  Returns
    (edges [NE, 2], face_cycles [NF, 4], cell_faces [nc, 6], cell_dofs [nc, 27]) with the cell DOF
    numbering of :3045-3054 (vertices, then NV + edge, NV + NE + face, NV + NE + NF + cell)."""
    cv = np.asarray(cell_vertex, dtype=np.int64)
    cyc = [tuple(int(g) for g in cv[c][FACE_CYCLES[f]]) for c in range(cv.shape[0]) for f in range(6)]
    faces = sorted(set(cyc))
    fid = {t: i for i, t in enumerate(faces)}
    pairs = sorted({(min(t[k], t[(k + 1) % 4]), max(t[k], t[(k + 1) % 4])) for t in faces for k in range(4)})
    eid = {p: i for i, p in enumerate(pairs)}
    nv = int(cv.max()) + 1
    ne, nf = len(pairs), len(faces)
    cell_faces = np.array([[fid[cyc[6 * c + f]] for f in range(6)] for c in range(cv.shape[0])])
    dofs = []
    for c in range(cv.shape[0]):
        es = sorted({eid[(min(t[k], t[(k + 1) % 4]), max(t[k], t[(k + 1) % 4]))]
                     for t in (faces[i] for i in cell_faces[c]) for k in range(4)})
        dofs.append(list(cv[c]) + [nv + e for e in es] + [nv + ne + f for f in cell_faces[c]] + [nv + ne + nf + c])
    return np.array(pairs), np.array(faces), cell_faces, np.array(dofs)


ORDER2_REF = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "order2_ref")


def macro_portrait(cell_dofs, n_dofs):
    """The Order2 macro portrait (Grid_forMech::CreationPortrait, MsFEM/MsFEM.h:53-55): DOF row d
    holds the DOFs sharing a cell with d, the diagonal included, ascending."""
    rows = [set() for _ in range(n_dofs)]
    for dl in np.asarray(cell_dofs):
        for d in dl:
            rows[int(d)].update(int(e) for e in dl)
    return [np.array(sorted(r), dtype=np.int64) for r in rows]


def run_reference(workdir, vertex_xyz, cell_vertex, cells, matrices=True, timeout=1200, groups=None,
                  min_residual=1e-13, order1=False):
    """Writes the macro mesh and cell directories under workdir (meshio writers), runs the
    reference's Order2 construction there and returns {"n": [ne, nv, n_edges, n_faces, n_dofs],
    "edges", "faces" (first-reached (id, n, edge ids...) records), "cell_dofs" [nc, 27],
    "cell_faces" [nc, 6], "bases" [per cell: (n_nodes, 27, 3)], "K" [per cell: (81, 81)],
    "solution" [n_dofs, 3] (groups given: the whole Order2 driver with those Dirichlet groups)}.
    order1=True (with groups): the Order1 driver instead (Grid_forMech_Poly_Order1,
    MsFEM_forElasticDeformation_OrderBF1_forPoly): "solution" [n_vertices, 3] and "bases" [per cell:
    (n_nodes, 8, 3)]."""
    import subprocess

    from multiscalefemsolver3d_b200 import meshio
    macro, fine, out = (os.path.join(workdir, p) for p in ("macro", "fine", "order2.bin"))
    meshio.write_macro_nvtr(macro, vertex_xyz, cell_vertex)
    meshio.write_cell_dirs(fine, cells)
    args = [ORDER2_REF, macro, fine, out, str(len(cells.E))]
    for e, n_ in zip(cells.E, cells.nu):
        args += [repr(float(e)), repr(float(n_))]
    if matrices:
        args.append("--matrices")
    if groups is not None:
        bc = os.path.join(workdir, "dirichlet.txt")
        with open(bc, "w") as fb:
            fb.write(f"{len(groups)}\n")
            for verts, value, take in groups:
                fb.write(" ".join(str(int(t)) for t in take) + " " + " ".join(repr(float(v)) for v in value) +
                         f" {len(verts)} " + " ".join(str(int(v)) for v in verts) + "\n")
        args += ["--driver", bc, repr(float(min_residual))]
        if order1:
            args.append("--order1")
    r = subprocess.run(args, stdin=subprocess.DEVNULL, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE,
                       timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"order2_ref failed ({r.returncode}): {r.stderr[-400:]!r}")
    raw = open(out, "rb").read()
    i, recs = 0, {}
    while i < len(raw):
        tag, cnt = (int(t) for t in np.frombuffer(raw, np.int32, 2, i))
        i += 8
        dt = np.float64 if tag in (5, 6) else np.int32
        a = np.frombuffer(raw, dt, cnt, i)
        i += cnt * np.dtype(dt).itemsize
        recs.setdefault(tag, []).append(a)
    if order1:
        # the Order1 construction writes its bases under <result dir>/tmp/Elem_<c> (MsFEM.h:597-605,
        # MsFEM_Grid.h:4808, :5556-5566)
        return {"solution": recs[6][0].reshape(-1, 3),
                "bases": [np.stack([np.loadtxt(os.path.join(fine, "tmp", f"Elem_{c}", f"BasisFunction_{b}.txt")).reshape(-1, 3)
                                    for b in range(8)], axis=1) for c in range(cells.n_cells)]}
    head = recs[1][0]
    nc = int(head[0])
    el = recs[4][0].reshape(nc, 1 + 27 + 6)
    res = {"n": head, "edges": recs[2][0].reshape(-1, 2), "faces": recs[3][0], "cell_dofs": el[:, 1:28],
           "cell_faces": el[:, 28:], "K": [k.reshape(81, 81) for k in recs.get(5, [])], "bases": [],
           "solution": recs[6][0].reshape(-1, 3) if 6 in recs else None,
           "portrait": recs[7][0] if 7 in recs else None}
    for c in range(nc):
        sub = os.path.join(fine, f"Elem_{c}", "SubElem_0")
        res["bases"].append(np.stack([np.loadtxt(os.path.join(sub, f"BasisFunction_{b}.txt")).reshape(-1, 3)
                                      for b in range(27)], axis=1))
    return res


def graded_cells(nc, m, grade, seed=1, contrast=10.0):
    """(macro vertex xyz, cell_vertex [nc^3, 8], CellMeshes): nc^3 box cells of the unit cube
    (meshgen.msfem_cells, ellipsoid inclusions), each cell's fine nodes moved along every axis by
    u -> u + grade (1 + 0.3 axis) sin(2 pi u) / (2 pi) in cell units (graded, non-uniform
    segments; the cell's faces and edges stay in place).  Graded edges keep the reference's edge
    solves from meeting MIN_RESIDUAL on their first pass."""
    from multiscalefemsolver3d_b200 import meshgen
    cm = meshgen.msfem_cells(n_coarse=nc, m_choices=(m,), seed=seed, contrast=contrast)
    for c in range(cm.n_cells):
        a, b = cm.node_off[c], cm.node_off[c + 1]
        for ax in range(3):
            lo, hi = cm.box[c][2 * ax], cm.box[c][2 * ax + 1]
            u = (cm.xyz[a:b, ax] - lo) / (hi - lo)
            g = u + grade * (1 + 0.3 * ax) * np.sin(2 * np.pi * u) / (2 * np.pi)
            g = np.where(np.abs(u) < 1e-14, 0.0, np.where(np.abs(u - 1) < 1e-14, 1.0, g))
            cm.xyz[a:b, ax] = lo + (hi - lo) * g
    s = np.arange(nc + 1) / nc
    kk, jj, ii = np.meshgrid(s, s, s, indexing="ij")
    vxyz = np.stack([ii.ravel(), jj.ravel(), kk.ravel()], axis=1)
    cv = np.array([[(c % nc + (b & 1)) + (nc + 1) * ((c // nc % nc + (b >> 1 & 1)) + (nc + 1) * (c // nc ** 2 + (b >> 2 & 1)))
                    for b in range(8)] for c in range(nc ** 3)])
    return vxyz, cv, cm


# --------------------------------------------------------------------------------------------
# The Order2 macro driver (MsFEM/MsFEM.h:14-569)
# --------------------------------------------------------------------------------------------

def polygon_rule3(V):
    """geometry::Polygon::SetIntegrationLaw(3) (Library/GeometryShape.h:2625-2640): the fan of
    triangles (centroid, V_i, V_i+1), each with Triangle::SetIntegrationLaw(3) (:1482-1540) as
    written there: weights 1/6 |e1 x e2| at (1/6, 1/6), (2/3, 1/6) and again (2/3, 1/6) -- its third
    point repeats the second where the symmetric rule has (1/6, 2/3)."""
    V = np.asarray(V, dtype=np.float64)
    C = V.mean(axis=0)
    pts, w = [], []
    for i in range(V.shape[0]):
        e1, e2 = V[i] - C, V[(i + 1) % V.shape[0]] - C
        det = np.linalg.norm(np.cross(e1, e2))
        for a, b in ((1 / 6, 1 / 6), (2 / 3, 1 / 6), (2 / 3, 1 / 6)):
            pts.append(C + a * e1 + b * e2)
            w.append(det / 6.0)
    return np.array(pts), np.array(w)


def _basis_at(xyz, tets, bases, I, x):
    """z component of basis I at x, from the micro tetrahedron holding x (the nearest-element
    lookup and P1 interpolation of the reference's macro basis functions, :2942-2950)."""
    e = oc.locate(xyz, tets, x)
    P = xyz[tets[e]]
    lam = np.linalg.solve((P[1:] - P[0]).T, x - P[0])
    bary = np.concatenate([[1 - lam.sum()], lam])
    return float(bary @ bases[tets[e], I, 2])


def order2_driver(vertex_xyz, cell_vertex, cells, groups, bases=None):
    """The Order2 macro solution [n_dofs, 3] (MsFEM_forElasticDeformation_OrderBF2_forPoly):
    groups = [(vertex ids, value (3,), take (3 bools))], the Dirichlet groups.  Steps:
      * bases and macro element matrices of every cell (order2_bases, macro_element_matrix), D of
        domain 0, summed into the 3x3-block system by the cells' DOF lists (macro_topology);
      * per group (Grid_forMech::CreateBoundaryConditions, MsFEM_Grid.h:3303-3470): its DOFs (the
        vertices, the edges with both ends in it, the faces with all vertices in it, ascending),
        the L2 projection of its value onto them over its faces -- the mass matrix and load of the
        faces' 9 DOFs (4 vertices, 4 edges, the face) with the polygon rule 3, the bases' z
        components evaluated in the face's first element -- solved per component (the face
        bubbles vanish on their faces: their values are 0);
      * the scalar copy of the system (DOF 3 d + c), and for every group DOF in order, every taken
        component: X = F = value, the row set to the identity and the column moved to F
        (MsFEM.h:300-365);
      * no Neumann data: the Order2 grid builds no boundary faces, so the loop at MsFEM.h:54-59 adds
        nothing;
      * the solve (here exact; the reference runs plain CG restarts, MsFEM.h:445-478).
    bases: optional precomputed [per cell (n_nodes, 27, 3)]."""
    edges, faces, cell_faces, dofs = macro_topology(cell_vertex)
    vertex_xyz = np.asarray(vertex_xyz, dtype=np.float64)
    nv, ne, nf = vertex_xyz.shape[0], len(edges), len(faces)
    nd = nv + ne + nf + len(cell_vertex)
    if bases is None:
        bases = []
        for c in range(cells.n_cells):
            xyz, tets, mat, box = cells.cell(c)
            bases.append(order2_bases(xyz, tets, mat, box, cells.E, cells.nu, cell_vertex[c]))
    A = np.zeros((3 * nd, 3 * nd))
    for c in range(cells.n_cells):
        xyz, tets, mat, box = cells.cell(c)
        K = macro_element_matrix(xyz, tets, bases[c], box, cells.E[0], cells.nu[0])
        idx = (3 * dofs[c][:, None] + np.arange(3)).ravel()
        A[np.ix_(idx, idx)] += K.transpose(0, 2, 1, 3).reshape(81, 81)
    fixed = dirichlet_fixed(vertex_xyz, cell_vertex, cells, groups, bases)
    F = np.zeros(3 * nd)
    for i, val in fixed:
        col = A[:, i].copy()
        col[i] = 0.0
        F -= col * val
        A[:, i] = 0.0
        A[i, :] = 0.0
        A[i, i] = 1.0
        F[i] = val
    return np.linalg.solve(A, F).reshape(nd, 3)


def dirichlet_fixed(vertex_xyz, cell_vertex, cells, groups, bases):
    """[(scalar DOF, value)] of the Order2 Dirichlet groups in the reference's order (the
    projection step of order2_driver)."""
    edges, faces, cell_faces, dofs = macro_topology(cell_vertex)
    vertex_xyz = np.asarray(vertex_xyz, dtype=np.float64)
    nv, ne, nf = vertex_xyz.shape[0], len(edges), len(faces)
    # the first element of each face (faces shared by two cells are interior, never Dirichlet)
    face_cell = {}
    for c in range(len(cell_vertex)):
        for f in cell_faces[c]:
            face_cell.setdefault(int(f), c)
    eid = {tuple(p): i for i, p in enumerate(edges)}
    fixed = []                                       # (scalar DOF, value) in the reference's order
    for verts, value, take in groups:
        vs = [int(v) for v in verts]
        sv = set(vs)
        gd = list(vs)
        gd += [nv + i for i, (a, b) in enumerate(edges) if a in sv and b in sv]
        tf = [i for i in range(nf) if set(int(v) for v in faces[i]) <= sv]
        gd += [nv + ne + i for i in tf]
        gd = sorted(gd)
        pos = {d: k for k, d in enumerate(gd)}
        M = np.zeros((len(gd), len(gd)))
        Fg = np.zeros((len(gd), 3))
        for f in tf:
            cyc = [int(v) for v in faces[f]]
            fd = cyc + [nv + eid[(min(cyc[k], cyc[(k + 1) % 4]), max(cyc[k], cyc[(k + 1) % 4]))] for k in range(4)]
            fd += [nv + ne + f]
            c = face_cell[f]
            xyz, tets, mat, box = cells.cell(c)
            loc = {int(d): k for k, d in enumerate(dofs[c])}
            pts, w = polygon_rule3(vertex_xyz[cyc])
            psi = np.array([[_basis_at(xyz, tets, bases[c], loc[d], x) for d in fd] for x in pts])   # [q, 9]
            Ml = np.einsum("q,qi,qj->ij", w, psi, psi)
            Fl = np.einsum("q,qi->i", w, psi)[:, None] * np.asarray(value, dtype=np.float64)[None, :]
            for I, di in enumerate(fd):
                if di not in pos:
                    continue
                for J, dj in enumerate(fd):
                    if dj in pos:
                        M[pos[di], pos[dj]] += Ml[I, J]
                Fg[pos[di]] += Fl[I]
        # the face bubble vanishes on its own face (its face problem has no load), so its row and
        # column of M are zero; the reference's Gauss leaves 0 there, as the least-squares solve does
        vals = np.linalg.lstsq(M, Fg, rcond=None)[0]
        for k, d in enumerate(gd):
            for comp in range(3):
                if take[comp]:
                    fixed.append((3 * d + comp, vals[k, comp]))
    return fixed
