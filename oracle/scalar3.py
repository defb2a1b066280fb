"""Test infrastructure only: CPU restatement of the reference's three-coefficient scalar FEM
(FiniteElement_forScal::SolveLocalMatrix with stiffness, mass and source coefficients,
FEM/FEM_Grid.h:25-102, and its driver FEM::FEM_forBaseEliptic, FEM/FEM.h:206-397).

Per tetrahedron, with the one-point rule (the centroid, weight V: Tetrahedron::SetIntegrationLaw(1),
Library/GeometryShape.h:1754-1762) and the coefficients S, M, f of the element:
    A_ij = V (S grad(phi_i).grad(phi_j) + M phi_i phi_j) = V (S g_i.g_j + M / 16),
    F_i  = V f phi_i = V f / 4;
summed into the node portrait (SummPartOfMatrix adds F too, Library/CSSD_Matrix.h:307-360), then
Dirichlet rows only (X = F = value, the row set to the identity, the columns left,
FEM.h:291-310), solved here exactly (the reference runs BiCG_Stab restarts to MIN_RESIDUAL)."""
from __future__ import annotations

import numpy as np


def local(P, S, M, f):
    """(A [4, 4], F [4]) of one tetrahedron P [4, 3]."""
    P = np.asarray(P, dtype=np.float64)
    E = (P[1:] - P[0]).T
    Ginv = np.linalg.inv(E)                                     # rows: gradients of l1..l3
    g = np.vstack([-Ginv.sum(axis=0), Ginv])
    V = abs(np.linalg.det(E)) / 6.0
    return V * (S * (g @ g.T) + M / 16.0), np.full(4, V * f / 4.0)


def driver(xyz, tets, S, M, f, bc_nodes, bc_values):
    """The driver's solution [n_nodes] (later duplicates of a Dirichlet node win)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spl
    xyz = np.asarray(xyz, dtype=np.float64)
    tets = np.asarray(tets, dtype=np.int64)
    n = xyz.shape[0]
    rows, cols, vals = [], [], []
    F = np.zeros(n)
    for e, t in enumerate(tets):
        A, Fe = local(xyz[t], S[e], M[e], f[e])
        rows.append(np.repeat(t, 4))
        cols.append(np.tile(t, 4))
        vals.append(A.ravel())
        np.add.at(F, t, Fe)
    K = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n)).tolil()
    for v, val in zip(bc_nodes, bc_values):
        K.rows[v] = [v]
        K.data[v] = [1.0]
        F[v] = val
    return spl.spsolve(K.tocsc(), F)
