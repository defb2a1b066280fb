"""Thermal conduction with insulating disc cracks by Heaviside enrichment (XFEM), scalar P1 on
Kuhn tetrahedra -- the workload of the 96^3 cracked-cube configuration.

The reference's XFEM is for elasticity only (MultiXFEM/MultiXFEM_Grid.h:1090-2980); this is the
scalar counterpart, restated with the same ingredients:

* crack k: a disc (centre c_k, unit normal n_k, radius r_k); d_k(x) = n_k . (x - c_k);
  H_k(x) = +1 where d_k >= 0, -1 elsewhere;
* a tetrahedron is cut by crack k when its vertices' d_k take both signs (strictly) and the
  projection of its centroid on the crack plane lies within r_k of c_k; a tetrahedron cut by
  several cracks takes the lowest-numbered one;
* every (vertex of a cut tetrahedron, its crack) pair carries an enriched DOF whose basis is the
  shifted Heaviside function psi = phi_v (H_k - H_k(x_v)), supported on the tetrahedra cut by k;
* on a cut tetrahedron with side volumes V+ and V- (exact plane clipping, `side_fraction`) and
  K_ij = sigma grad(phi_i) . grad(phi_j):  std-std = (V+ + V-) K_ij, std(i)-enr(j) =
  sum_s V_s (H_s - H_j) K_ij, enr(i)-enr(j) = sum_s V_s (H_s - H_i)(H_s - H_j) K_ij.  No flux
  crosses the crack (insulating): nothing couples the two sides across it.

DOFs: nodes 0..N-1, then the enriched DOFs in (crack, node) order.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import meshgen

__all__ = ["Cracks", "Enrichment", "random_cracks", "enrich", "side_fraction", "cube_cracked", "build_system"]


@dataclass
class Cracks:
    centre: np.ndarray   # [k, 3]
    normal: np.ndarray   # [k, 3] unit
    radius: np.ndarray   # [k]


@dataclass
class Enrichment:
    n_dofs: int                 # nodes + enriched DOFs
    crack_of_tet: np.ndarray    # int32 [n_tets], -1 = not cut
    enr_dof: np.ndarray         # int32 [n_tets, 4]: enriched DOF of each vertex (-1 when not cut)
    n_enriched: int


def random_cracks(count: int, rmin: float, rmax: float, seed: int) -> Cracks:
    """Centres U(0,1)^3, normals uniform on the sphere, radii U(rmin, rmax), in draw order."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(0.0, 1.0, size=(count, 3))
    n = rng.normal(size=(count, 3))
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    r = rng.uniform(rmin, rmax, size=count)
    return Cracks(c, n, r)


def side_fraction(d):
    """Volume fraction of a tetrahedron where the linear function with vertex values d (..., 4)
    is >= 0, exactly: one vertex on the + side: d_a^3 / prod(d_a - d_j); three: one minus the
    same for the - vertex; two (a, b | c, e): the divided difference with the (d_a - d_b) factor
    taken out, (d_a^2 d_b^2 - p d_a d_b (d_a + d_b) + q (d_a^2 + d_a d_b + d_b^2)) /
    ((d_a - d_c)(d_a - d_e)(d_b - d_c)(d_b - d_e)), p = d_c + d_e, q = d_c d_e."""
    d = np.asarray(d, dtype=np.float64)
    pos = d >= 0.0
    k = pos.sum(axis=-1)
    out = np.where(k == 4, 1.0, 0.0).astype(np.float64)
    flat_d = d.reshape(-1, 4)
    flat_k = k.reshape(-1)
    res = out.reshape(-1)
    for i in np.nonzero((flat_k > 0) & (flat_k < 4))[0]:
        res[i] = _frac1(flat_d[i])
    return res.reshape(out.shape)


def _frac1(d):
    P = [v for v in range(4) if d[v] >= 0.0]
    M = [v for v in range(4) if d[v] < 0.0]
    if len(P) == 1:
        a = P[0]
        den = 1.0
        for j in M:
            den *= d[a] - d[j]
        return d[a] ** 3 / den
    if len(P) == 3:
        b = M[0]
        den = 1.0
        for j in P:
            den *= d[j] - d[b]
        return 1.0 - (-d[b]) ** 3 / den
    a, b = P
    c, e = M
    p, q = d[c] + d[e], d[c] * d[e]
    num = d[a] ** 2 * d[b] ** 2 - p * d[a] * d[b] * (d[a] + d[b]) + q * (d[a] ** 2 + d[a] * d[b] + d[b] ** 2)
    return num / ((d[a] - d[c]) * (d[a] - d[e]) * (d[b] - d[c]) * (d[b] - d[e]))


def enrich(xyz, tets, cracks: Cracks) -> Enrichment:
    """Cut tetrahedra, their cracks and the enriched DOF numbering (module docstring)."""
    xyz = np.asarray(xyz, dtype=np.float64)
    tets = np.asarray(tets, dtype=np.int64)
    n_nodes, n_tets = xyz.shape[0], tets.shape[0]
    crack_of = -np.ones(n_tets, np.int64)
    P = xyz[tets]
    cen = P.mean(axis=1)
    # a tetrahedron the plane crosses has |centroid - plane| <= its diameter, so a cut one lies
    # within radius + diameter of the centre: test only those
    ea, eb = [0, 0, 0, 1, 1, 2], [1, 2, 3, 2, 3, 3]
    diam = float(np.sqrt(((P[:, ea] - P[:, eb]) ** 2).sum(-1).max())) if n_tets else 0.0
    del P
    # centroids bucketed by z so that each crack scans only the slab it can reach
    order = np.argsort(cen[:, 2], kind="stable")
    zs = cen[order, 2]
    for k in range(cracks.radius.size):
        reach = cracks.radius[k] + diam
        lo, hi = np.searchsorted(zs, cracks.centre[k][2] - reach), np.searchsorted(zs, cracks.centre[k][2] + reach)
        cand = np.sort(order[lo:hi])
        near = cand[((cen[cand] - cracks.centre[k]) ** 2).sum(axis=1) < reach ** 2]
        if near.size == 0:
            continue
        dt = (xyz[tets[near]] - cracks.centre[k]) @ cracks.normal[k]
        cut = (dt.max(axis=1) > 0.0) & (dt.min(axis=1) < 0.0) & (crack_of[near] < 0)
        idx = near[cut]
        if idx.size == 0:
            continue
        rel = cen[idx] - cracks.centre[k]
        inplane = rel - np.outer(rel @ cracks.normal[k], cracks.normal[k])
        inside = np.einsum("ij,ij->i", inplane, inplane) < cracks.radius[k] ** 2
        crack_of[idx[inside]] = k
    cut_tets = np.nonzero(crack_of >= 0)[0]
    pairs = np.stack([np.repeat(crack_of[cut_tets], 4), tets[cut_tets].ravel()], axis=1)  # (crack, node)
    key = pairs[:, 0] * n_nodes + pairs[:, 1]
    uniq, inv = np.unique(key, return_inverse=True)
    enr = -np.ones((n_tets, 4), np.int64)
    enr[cut_tets] = (n_nodes + inv).reshape(-1, 4)
    return Enrichment(n_dofs=n_nodes + uniq.size, crack_of_tet=crack_of.astype(np.int32),
                      enr_dof=enr.astype(np.int32), n_enriched=int(uniq.size))


def cube_cracked(n: int = 96, n_cracks: int = 50, seed: int = 5, rmin: float = 0.03, rmax: float = 0.1):
    """The cracked-cube workload: kuhn_cube(n), conductivity 1, T = 1 on z = 0 and 0 on z = 1,
    n_cracks seeded disc cracks.  Returns (mesh, cracks, Dirichlet nodes, values)."""
    mesh = meshgen.kuhn_cube(n)
    cracks = random_cracks(n_cracks, rmin, rmax, seed)
    lo = meshgen.nodes_on_plane(mesh, 2, 0.0)
    hi = meshgen.nodes_on_plane(mesh, 2, 1.0)
    nodes = np.concatenate([lo, hi]).astype(np.int32)
    vals = np.concatenate([np.ones(lo.size), np.zeros(hi.size)])
    return mesh, cracks, nodes, vals


def build_system(mesh, cracks: Cracks, sigma=1.0, enr: Enrichment | None = None):
    """(fem.System of the enriched problem assembled on the GPU (msfem_xfem_system), Enrichment)."""
    import ctypes as C

    from . import fem
    from ._lib import check, load
    enr = enrich(mesh.xyz, mesh.tets, cracks) if enr is None else enr
    xyz = np.ascontiguousarray(mesh.xyz, dtype=np.float64)
    tets = np.ascontiguousarray(mesh.tets, dtype=np.int32)
    sig = np.ascontiguousarray(np.broadcast_to(np.asarray(sigma, dtype=np.float64), (tets.shape[0],)))
    cen = np.ascontiguousarray(cracks.centre, dtype=np.float64)
    nor = np.ascontiguousarray(cracks.normal, dtype=np.float64)
    cof = np.ascontiguousarray(enr.crack_of_tet, dtype=np.int32)
    edf = np.ascontiguousarray(enr.enr_dof, dtype=np.int32)
    P = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    h = C.c_void_p()
    check(load().msfem_xfem_system(xyz.shape[0], P(xyz), tets.shape[0], P(tets), P(sig), cen.shape[0], P(cen), P(nor),
                                   P(cof), P(edf), enr.n_dofs, C.byref(h)), "xfem_system")
    return fem.System._from_handle(h), enr
