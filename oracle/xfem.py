"""Test infrastructure only: CPU restatement (numpy/scipy) of the cracked-conduction assembly of
multiscalefemsolver3d_b200/xfem.py and csrc/xfem.cu -- standard P1 stiffness sigma V
grad(phi_i) . grad(phi_j) on every tetrahedron, plus the shifted-Heaviside enriched blocks on cut
tetrahedra weighted by the exact side volumes.  The reference has no scalar XFEM, so nothing of
the reference pins this; tests/test_xfem_oracle.py checks it against exact answers (a crack
through the whole cube decouples the two halves; no crack reproduces the plain assembly).

Independent of the product's host code: the side volumes come from geometric clipping
(clip_fraction: the tetrahedron cut by the plane, the positive part assembled from small
tetrahedra) rather than the product's closed-form fractions, and the cut detection and enriched
numbering are restated as plain loops (enrich)."""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp


def _tet_volume(a, b, c, d):
    return abs(np.dot(b - a, np.cross(c - a, d - a))) / 6.0


def clip_fraction(P, d):
    """Volume fraction of the tetrahedron P [4, 3] where the linear function with vertex values
    d [4] is >= 0, from the clipped polytope itself: the edge crossings x_ab = P_a + t (P_b - P_a),
    t = d_a / (d_a - d_b), then one positive vertex: the corner tetrahedron; three: the whole minus
    the negative corner; two (a, b | c, e): the wedge a b x_ac x_ae x_bc x_be split into three
    tetrahedra."""
    P = np.asarray(P, dtype=np.float64)
    d = np.asarray(d, dtype=np.float64)
    V = _tet_volume(*P)
    pos = [i for i in range(4) if d[i] >= 0.0]
    neg = [i for i in range(4) if d[i] < 0.0]
    if not neg:
        return 1.0
    if not pos:
        return 0.0

    def x(a, b):
        return P[a] + d[a] / (d[a] - d[b]) * (P[b] - P[a])
    if len(pos) == 1:
        a = pos[0]
        return _tet_volume(P[a], *(x(a, j) for j in neg)) / V
    if len(pos) == 3:
        b = neg[0]
        return 1.0 - _tet_volume(P[b], *(x(b, j) for j in pos)) / V
    a, b = pos
    c, e = neg
    xac, xae, xbc, xbe = x(a, c), x(a, e), x(b, c), x(b, e)
    vol = _tet_volume(P[a], xac, xae, P[b]) + _tet_volume(P[b], xac, xae, xbe) + _tet_volume(P[b], xac, xbe, xbc)
    return vol / V


@dataclass
class Enrichment:
    n_dofs: int
    crack_of_tet: np.ndarray
    enr_dof: np.ndarray
    n_enriched: int


def enrich(xyz, tets, cracks):
    """Cut detection and enriched numbering, tetrahedron by tetrahedron: a tetrahedron is cut by
    crack k when its vertices' signed distances take both signs strictly and its centroid's
    projection on the plane lies within the radius; the lowest such k wins.  Enriched DOFs: the
    distinct (crack, node) pairs of the cut tetrahedra in ascending (crack, node) order, numbered
    from n_nodes."""
    xyz = np.asarray(xyz, np.float64)
    tets = np.asarray(tets, np.int64)
    n = xyz.shape[0]
    crack_of = -np.ones(tets.shape[0], np.int64)
    for e, t in enumerate(tets):
        P = xyz[t]
        cen = P.mean(axis=0)
        for k in range(len(cracks.radius)):
            dist = (P - cracks.centre[k]) @ cracks.normal[k]
            if not (dist.max() > 0.0 and dist.min() < 0.0):
                continue
            rel = cen - cracks.centre[k]
            inplane = rel - (rel @ cracks.normal[k]) * cracks.normal[k]
            if inplane @ inplane < cracks.radius[k] ** 2:
                crack_of[e] = k
                break
    pairs = sorted({(int(crack_of[e]), int(v)) for e in np.nonzero(crack_of >= 0)[0] for v in tets[e]})
    num = {p: n + i for i, p in enumerate(pairs)}
    enr = -np.ones((tets.shape[0], 4), np.int64)
    for e in np.nonzero(crack_of >= 0)[0]:
        enr[e] = [num[(int(crack_of[e]), int(v))] for v in tets[e]]
    return Enrichment(n + len(pairs), crack_of.astype(np.int32), enr.astype(np.int32), len(pairs))


def _grads(P):
    """[E, 4, 3] gradients of the barycentric functions and [E] volumes."""
    e1, e2, e3 = P[:, 1] - P[:, 0], P[:, 2] - P[:, 0], P[:, 3] - P[:, 0]
    c23, c31, c12 = np.cross(e2, e3), np.cross(e3, e1), np.cross(e1, e2)
    det = np.einsum("ij,ij->i", e1, c23)
    g = np.stack([np.zeros_like(e1), c23 / det[:, None], c31 / det[:, None], c12 / det[:, None]], axis=1)
    g[:, 0] = -(g[:, 1] + g[:, 2] + g[:, 3])
    return g, np.abs(det) / 6.0


def assemble(xyz, tets, sigma_tet, cracks, enr):
    """Global matrix (scipy CSR, n_dofs x n_dofs) of the enriched conduction problem."""
    xyz = np.asarray(xyz, np.float64)
    tets = np.asarray(tets, np.int64)
    g, V = _grads(xyz[tets])
    K = np.einsum("eid,ejd->eij", g, g) * (np.asarray(sigma_tet) * V)[:, None, None]   # [E,4,4] full volume
    rows = [np.repeat(tets, 4, axis=1).ravel()]
    cols = [np.tile(tets, (1, 4)).ravel()]
    vals = [K.ravel()]
    cut = np.nonzero(enr.crack_of_tet >= 0)[0]
    if cut.size:
        k = enr.crack_of_tet[cut]
        d = np.einsum("evd,ed->ev", xyz[tets[cut]] - cracks.centre[k][:, None, :], cracks.normal[k])
        fp = np.array([clip_fraction(xyz[tets[c]], dc) for c, dc in zip(cut, d)])
        H = np.where(d >= 0.0, 1.0, -1.0)                        # H at the vertices
        Kc = K[cut] / V[cut][:, None, None]                        # per unit volume
        Vp, Vm = fp * V[cut], (1.0 - fp) * V[cut]
        # std(i)-enr(j): sum_s V_s (H_s - H_j) K_ij ; enr(i)-enr(j): sum_s V_s (H_s - H_i)(H_s - H_j) K_ij
        wse = Vp[:, None, None] * (1.0 - H[:, None, :]) + Vm[:, None, None] * (-1.0 - H[:, None, :])
        wee = (Vp[:, None, None] * (1.0 - H[:, :, None]) * (1.0 - H[:, None, :])
               + Vm[:, None, None] * (-1.0 - H[:, :, None]) * (-1.0 - H[:, None, :]))
        se = Kc * wse
        ee = Kc * wee
        T = tets[cut]
        Ed = enr.enr_dof[cut].astype(np.int64)
        rows += [np.repeat(T, 4, axis=1).ravel(), np.repeat(Ed, 4, axis=1).ravel(), np.repeat(Ed, 4, axis=1).ravel()]
        cols += [np.tile(Ed, (1, 4)).ravel(), np.tile(T, (1, 4)).ravel(), np.tile(Ed, (1, 4)).ravel()]
        vals += [se.ravel(), np.transpose(se, (0, 2, 1)).ravel(), ee.ravel()]
    A = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(enr.n_dofs, enr.n_dofs)).tocsr()
    A.sum_duplicates()
    return A


def solve_dirichlet(A, nodes, values):
    """Exact solution with the Dirichlet DOFs eliminated (later duplicates win)."""
    import scipy.sparse.linalg as spl
    n = A.shape[0]
    x = np.zeros(n)
    fixed = np.zeros(n, bool)
    for v, val in zip(nodes, values):
        x[v] = val
        fixed[v] = True
    free = ~fixed
    A = A.tocsr()
    rhs = -A[free][:, fixed] @ x[fixed]
    x[free] = spl.spsolve(A[free][:, free].tocsc(), rhs)
    return x


def solve_dirichlet_gmres(A, nodes, values, tol=1e-8, restart=50, maxiter=200000):
    """The same eliminated system solved by restarted GMRES(restart) with Jacobi preconditioning
    (scipy), to ||r|| <= tol ||b|| of the eliminated system; returns (x, iterations)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    n = A.shape[0]
    x = np.zeros(n)
    fixed = np.zeros(n, bool)
    for v, val in zip(nodes, values):
        x[v] = val
        fixed[v] = True
    free = ~fixed
    A = A.tocsr()
    Aff = A[free][:, free].tocsr()
    rhs = -A[free][:, fixed] @ x[fixed]
    M = sp.diags(1.0 / Aff.diagonal())
    count = [0]

    def cb(_):
        count[0] += 1
    y, info = spl.gmres(Aff, rhs, M=M, rtol=tol, atol=0.0, restart=restart, maxiter=maxiter,
                        callback=cb, callback_type="pr_norm")
    x[free] = y
    return x, count[0]
