"""Test infrastructure only: CPU restatement of the two-level preconditioner built on the
MsFEM coarse space (multiscalefemsolver3d_b200/csrc/twolevel.cu), for checking the GPU's
prolongation, coarse Galerkin matrix and preconditioner application.

  P[(g, a), (V, a)] = mean over the cells c holding fine node g of psi_{c,V}^a(g)  (the Order1
                      basis of vertex V in cell c, its a-component), 0 on fine Dirichlet DOFs;
                      coarse DOFs (V, a) whose vertex node has a Dirichlet a-component dropped;
                      a cell with any basis value outside [-3, 3] (the reference's indefinite
                      cell operator near singularity) contributes the trilinear functions of its
                      box instead
  A_c = P^T K P,     K = the textbook orientation of the fine element blocks (SPD on the free DOFs)
  M^-1 r = r + S^-1 P A_c^-1 P^T S^-1 r   on the Jacobi-scaled system (S = diag(A)^-1/2)
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from . import cells as oc


WILD_BASIS = 3.0


def sanitized_bases(cc, bases):
    """Bases with every wild cell (|psi| > WILD_BASIS somewhere) replaced by the trilinear
    functions of its box, as the GPU's coarse build does."""
    cm = cc.cells
    out = np.array(bases, dtype=np.float64, copy=True)
    for c in range(cm.n_cells):
        a0, a1 = cm.node_off[c], cm.node_off[c + 1]
        if np.all(np.abs(out[a0:a1]) <= WILD_BASIS):
            continue
        box = cm.box[c]
        t = (cm.xyz[a0:a1] - box[[0, 2, 4]]) / (box[[1, 3, 5]] - box[[0, 2, 4]])
        for v in range(8):
            q = np.ones(a1 - a0)
            for d in range(3):
                q *= t[:, d] if (v >> d) & 1 else 1.0 - t[:, d]
            out[a0:a1, v, :] = q[:, None]
    return out


def prolongation(cc, bases, n_fine, fixed_dofs):
    """cc: meshgen.CubeCells; bases: [cells' nodes, 8, 3] (cell-local) -> (P [3 n_fine, n_cf] CSR,
    coarse_dof [n_cells, 8, 3] (-1 dropped))."""
    fixed = np.zeros(3 * n_fine, bool)
    fixed[np.asarray(fixed_dofs)] = True
    bases = sanitized_bases(cc, bases)
    cm = cc.cells
    n_cv = cc.n_coarse_vertices
    # coarse DOFs
    vfix = np.zeros((n_cv, 3), bool)
    for c in range(cm.n_cells):
        xyz, _, _, box = cm.cell(c)
        mask = oc.face_masks(xyz, box)
        for v in range(8):
            want = sum(1 << f for f in oc.vertex_faces(v))
            node = cm.node_off[c] + np.nonzero((mask & want) == want)[0][0]
            g = cc.cell_node_global[node]
            vfix[cc.cell_vertex[c, v]] = fixed[3 * g:3 * g + 3]
    dof = -np.ones(3 * n_cv, np.int64)
    free = ~vfix.ravel()
    dof[free] = np.arange(free.sum())
    n_cf = int(free.sum())
    # accumulate P (fine node, component) x (coarse vertex, component)
    acc = {}
    mult = np.bincount(cc.cell_node_global, minlength=n_fine)
    for c in range(cm.n_cells):
        a0, a1 = cm.node_off[c], cm.node_off[c + 1]
        g = cc.cell_node_global[a0:a1]
        B = bases[a0:a1]
        for v in range(8):
            V = cc.cell_vertex[c, v]
            for a in range(3):
                d = dof[3 * V + a]
                if d < 0:
                    continue
                vals = B[:, v, a] / mult[g]
                for gi, val in zip(g, vals):
                    if val != 0.0 and not fixed[3 * gi + a]:
                        key = (3 * gi + a, d)
                        acc[key] = acc.get(key, 0.0) + val
    rows = np.array([k[0] for k in acc], dtype=np.int64)
    cols = np.array([k[1] for k in acc], dtype=np.int64)
    P = sp.csr_matrix((np.array(list(acc.values())), (rows, cols)), shape=(3 * n_fine, n_cf))
    cdof = dof[3 * cc.cell_vertex[:, :, None] + np.arange(3)[None, None, :]]
    return P, cdof


def coarse_matrix(mesh, E, nu, P):
    K = oc.assemble(mesh.xyz, mesh.tets, mesh.mat, E, nu, textbook=True)
    Ac = (P.T @ K @ P).toarray()
    return 0.5 * (Ac + Ac.T)


def apply(A_fine_diag, P, Ac, r):
    s = 1.0 / np.sqrt(A_fine_diag)
    Ph = sp.diags(1.0 / s) @ P
    return r + Ph @ np.linalg.solve(Ac, Ph.T @ r)
