"""Test infrastructure only: CPU restatement (numpy/scipy) of the cracked-conduction assembly of
multiscalefemsolver3d_b200/xfem.py and csrc/xfem.cu -- standard P1 stiffness sigma V
grad(phi_i) . grad(phi_j) on every tetrahedron, plus the shifted-Heaviside enriched blocks on cut
tetrahedra weighted by the exact side volumes.  The reference has no scalar XFEM, so nothing of
the reference pins this; tests/test_xfem_oracle.py checks it against exact answers (a crack
through the whole cube decouples the two halves; no crack reproduces the plain assembly)."""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from multiscalefemsolver3d_b200.xfem import side_fraction


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
        fp = side_fraction(d)
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
