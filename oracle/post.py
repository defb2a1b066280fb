"""Test infrastructure only: CPU restatement of the elasticity post-processing.

Per element at its centroid (FEM/FEM_Grid.h:3289-3365): U = the P1 interpolant (the mean of the
nodal values), dU (row a = grad u_a), the strain tensor EPS (symmetric part of dU), the stress
tensor of the element's own material through the Voigt product of Domain::forMech::solve_SIGMA
(Library/Domain.h:231-290: [e_xx, e_yy, e_zz, 2 e_yz, 2 e_xz, 2 e_xy] times the isotropic D),
and GetVonMisesStress's formula (FEM_Grid.h:3361-3365: sqrt(sum of squared normal differences +
6 (s_xy s_yx + s_xz s_zx + s_yz s_zy) / 2)).  The driver's printed fields (FEM/FEM_Main.cpp:
1018-1040): domain 0's E and nu for every element, engineering shear strains, shear stresses
k 2 b gamma, and its own von Mises line.
"""
from __future__ import annotations

import numpy as np

from . import cells as oc


def element_fields(xyz, tets, mat, E, nu, u):
    """[n_tets, 23]: U(3), dU(9), sigma (xx yy zz yz xz xy), von Mises, then the driver's
    sigma_xx, sigma_yy, sigma_zz and von Mises."""
    xyz = np.asarray(xyz, np.float64)
    u = np.asarray(u, np.float64).reshape(-1, 3)
    out = np.zeros((len(tets), 23))
    D = [oc.isotropic_D(e, n) for e, n in zip(E, nu)]
    E0, v0 = float(E[0]), float(nu[0])
    a0, b0 = v0 / (1 - v0), (1 - 2 * v0) / (2 * (1 - v0))
    k0 = E0 * (1.0 - v0) / (1.0 + v0) / (1.0 - 2.0 * v0)
    for e, t in enumerate(np.asarray(tets)):
        P = xyz[t]
        G = np.linalg.inv(np.vstack([np.ones(4), P.T]))[:, 1:]      # rows: grad of barycentric j
        U = u[t].mean(axis=0)
        dU = u[t].T @ G                                              # [a][d] = d u_a / d x_d
        eps = 0.5 * (dU + dU.T)
        veps = np.array([eps[0, 0], eps[1, 1], eps[2, 2], 2 * eps[1, 2], 2 * eps[0, 2], 2 * eps[0, 1]])
        s = D[int(mat[e])] @ veps
        S = np.array([[s[0], s[5], s[4]], [s[5], s[1], s[3]], [s[4], s[3], s[2]]])
        vm = np.sqrt((S[0, 0] - S[1, 1]) ** 2 + (S[1, 1] - S[2, 2]) ** 2 + (S[0, 0] - S[2, 2]) ** 2
                     + 6 * (S[0, 1] * S[1, 0] + S[0, 2] * S[2, 0] + S[1, 2] * S[2, 1]) / 2.0)
        ed = [dU[0, 0], dU[1, 1], dU[2, 2], dU[0, 1] + dU[1, 0], dU[1, 2] + dU[2, 1], dU[0, 2] + dU[2, 0]]
        sd = [k0 * (ed[0] + ed[1] * a0 + ed[2] * a0), k0 * (ed[0] * a0 + ed[1] + ed[2] * a0),
              k0 * (ed[0] * a0 + ed[1] * a0 + ed[2]), k0 * 2 * ed[3] * b0, k0 * 2 * ed[4] * b0, k0 * 2 * ed[5] * b0]
        vmd = np.sqrt((sd[0] - sd[1]) ** 2 + (sd[1] - sd[2]) ** 2 + (sd[0] - sd[2]) ** 2
                      + 6 * (sd[3] ** 2 + sd[4] ** 2 + sd[5] ** 2) / 2.0)
        out[e, 0:3] = U
        out[e, 3:12] = dU.ravel()
        out[e, 12:18] = s
        out[e, 18] = vm
        out[e, 19:22] = sd[:3]
        out[e, 22] = vmd
    return out
