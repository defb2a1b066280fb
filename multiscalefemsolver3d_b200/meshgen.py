"""Seeded synthetic tetrahedral meshes for the solver's workloads.

The reference reads its meshes from NVTR/TecPlot files (Library/Math.h:150-291,
`math::SimpleGrid` = {nvtr, nvkat, xyz}, Library/Math.h:26-33).  These
generators build the same three arrays in memory:

  xyz   float64 [n_nodes, 3]   node coordinates
  tets  int32   [n_tets, 4]    node ids per tetrahedron (the reference's nvtr)
  mat   int32   [n_tets]       material / domain id per tetrahedron (nvkat)

Every hexahedron of an n x n x n grid on the unit cube is split into the six
Kuhn (Freudenthal) tetrahedra that share the cell diagonal 0-7, with corner b of
cell (i, j, k) at (i + (b & 1), j + ((b >> 1) & 1), k + ((b >> 2) & 1)) and node
id i + (n+1) * (j + (n+1) * k).  Interior nodes may be jittered by a seeded
uniform offset.  All randomness comes from numpy's PCG64 generator seeded
explicitly, so every workload is reproducible from its seed.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# corner sets of the six Kuhn tetrahedra of a hexahedron (corners 0..7 as above)
KUHN_TETS = np.array(
    [[0, 1, 3, 7], [0, 1, 5, 7], [0, 2, 3, 7], [0, 2, 6, 7], [0, 4, 5, 7], [0, 4, 6, 7]], dtype=np.int64
)


@dataclass
class Mesh:
    xyz: np.ndarray
    tets: np.ndarray
    mat: np.ndarray
    n: int = 0
    meta: dict = field(default_factory=dict)

    @property
    def n_nodes(self) -> int:
        return int(self.xyz.shape[0])

    @property
    def n_tets(self) -> int:
        return int(self.tets.shape[0])


def node_id(n: int, i, j, k):
    return i + (n + 1) * (j + (n + 1) * k)


def kuhn_cube(n: int, jitter: float = 0.0, seed: int = 0, origin=(0.0, 0.0, 0.0), size: float = 1.0) -> Mesh:
    """n^3 hexahedra on [origin, origin+size]^3, six Kuhn tets each.

    jitter: interior nodes move by U(-jitter*h, +jitter*h) per axis (h = size/n).
    """
    h = size / n
    g = np.arange(n + 1, dtype=np.float64)
    k, j, i = np.meshgrid(g, g, g, indexing="ij")  # node id = i + (n+1)(j + (n+1)k)
    xyz = np.stack([i.ravel() * h + origin[0], j.ravel() * h + origin[1], k.ravel() * h + origin[2]], axis=1)
    if jitter > 0.0:
        ii, jj, kk = i.ravel().astype(np.int64), j.ravel().astype(np.int64), k.ravel().astype(np.int64)
        interior = (ii > 0) & (ii < n) & (jj > 0) & (jj < n) & (kk > 0) & (kk < n)
        rng = np.random.default_rng(seed)
        off = rng.uniform(-jitter * h, jitter * h, size=(int(interior.sum()), 3))
        xyz[interior] += off
    c = np.arange(n, dtype=np.int64)
    ck, cj, ci = np.meshgrid(c, c, c, indexing="ij")
    ci, cj, ck = ci.ravel(), cj.ravel(), ck.ravel()
    corners = np.stack(
        [node_id(n, ci + (b & 1), cj + ((b >> 1) & 1), ck + ((b >> 2) & 1)) for b in range(8)], axis=1
    )  # [n^3, 8]
    tets = corners[:, KUHN_TETS].reshape(-1, 4).astype(np.int32)
    mat = np.zeros(tets.shape[0], dtype=np.int32)
    return Mesh(xyz=xyz, tets=tets, mat=mat, n=n, meta={"jitter": jitter, "seed": seed})


def nodes_on_plane(mesh: Mesh, axis: int, value: float, tol: float = 1e-12) -> np.ndarray:
    """Ids of nodes whose coordinate `axis` equals value, ascending."""
    return np.nonzero(np.abs(mesh.xyz[:, axis] - value) < tol)[0].astype(np.int32)


def boundary_faces_on_plane(mesh: Mesh, axis: int, value: float, tol: float = 1e-12):
    """Triangles of tets with three nodes on the plane: (faces [m,3], base element [m]).

    Face node order follows the tet's local node order, the way the reference's
    Neumann reader collects them (FEM/FEM_Main.cpp:819-872, GetConfluence order).
    """
    on = np.abs(mesh.xyz[:, axis] - value) < tol
    flags = on[mesh.tets]  # [E,4]
    hit = np.nonzero(flags.sum(axis=1) == 3)[0]
    faces = np.empty((hit.size, 3), dtype=np.int32)
    for r, e in enumerate(hit):
        faces[r] = mesh.tets[e][flags[e]]
    return faces, hit.astype(np.int32)


def tet_centroids(mesh: Mesh) -> np.ndarray:
    return mesh.xyz[mesh.tets].mean(axis=1)


def random_spheres(count: int, rmin: float, rmax: float, seed: int, max_tries: int = 1_000_000):
    """`count` non-overlapping spheres in the unit cube: centres U(0,1)^3,
    radii U(rmin, rmax), rejection-sampled in draw order."""
    rng = np.random.default_rng(seed)
    centres = np.empty((count, 3))
    radii = np.empty(count)
    m = 0
    tries = 0
    while m < count:
        tries += 1
        if tries > max_tries:
            raise RuntimeError(f"could only place {m} of {count} spheres")
        c = rng.uniform(0.0, 1.0, size=3)
        r = rng.uniform(rmin, rmax)
        if m and np.any(np.linalg.norm(centres[:m] - c, axis=1) < radii[:m] + r):
            continue
        centres[m] = c
        radii[m] = r
        m += 1
    return centres, radii


def mark_spheres(mesh: Mesh, centres: np.ndarray, radii: np.ndarray, material: int = 1) -> None:
    """Sets mat = material for every tet whose centroid lies inside a sphere.
    Only tets of the structured grid cells overlapping each sphere's bounding
    box are tested (the mesh must come from kuhn_cube on the unit cube)."""
    n = mesh.n
    cen = tet_centroids(mesh)
    for c, r in zip(centres, radii):
        lo = np.clip(np.floor((c - r) * n).astype(int) - 1, 0, n - 1)
        hi = np.clip(np.floor((c + r) * n).astype(int) + 1, 0, n - 1)
        ci = np.arange(lo[0], hi[0] + 1)
        cj = np.arange(lo[1], hi[1] + 1)
        ck = np.arange(lo[2], hi[2] + 1)
        kk, jj, ii = np.meshgrid(ck, cj, ci, indexing="ij")
        cells = (ii + n * (jj + n * kk)).ravel()
        tet_ids = (cells[:, None] * 6 + np.arange(6)[None, :]).ravel()
        inside = np.sum((cen[tet_ids] - c) ** 2, axis=1) < r * r
        mesh.mat[tet_ids[inside]] = material


# ----------------------------------------------------------------------------------------------
# Workloads (sizes and distributions of the synthetic configurations)
# ----------------------------------------------------------------------------------------------

@dataclass
class ElasticProblem:
    mesh: Mesh
    E: np.ndarray
    nu: np.ndarray
    bc_nodes: np.ndarray      # Dirichlet nodes (ascending)
    bc_mask: np.ndarray       # bit 0/1/2 = x/y/z component fixed
    bc_values: np.ndarray     # [m, 3]
    faces: np.ndarray         # traction triangles [f, 3]
    face_elem: np.ndarray     # base tetrahedron of each triangle
    traction: np.ndarray      # [f, 3]


def kuhn_box(nx: int, ny: int, nz: int, size=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0)) -> Mesh:
    """nx x ny x nz hexahedra on a box, six Kuhn tets each, in kuhn_cube's layout (node id
    i + (nx+1) (j + (ny+1) k), hexahedron i + nx (j + ny k))."""
    hx, hy, hz = size[0] / nx, size[1] / ny, size[2] / nz
    k, j, i = np.meshgrid(np.arange(nz + 1.0), np.arange(ny + 1.0), np.arange(nx + 1.0), indexing="ij")
    xyz = np.stack([i.ravel() * hx + origin[0], j.ravel() * hy + origin[1], k.ravel() * hz + origin[2]], axis=1)
    ck, cj, ci = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ci, cj, ck = ci.ravel(), cj.ravel(), ck.ravel()
    corners = np.stack([(ci + (b & 1)) + (nx + 1) * ((cj + ((b >> 1) & 1)) + (ny + 1) * (ck + ((b >> 2) & 1)))
                        for b in range(8)], axis=1)
    tets = corners[:, KUHN_TETS].reshape(-1, 4).astype(np.int32)
    return Mesh(xyz=xyz, tets=tets, mat=np.zeros(tets.shape[0], dtype=np.int32), n=nx,
                meta={"box": (nx, ny, nz), "size": tuple(size)})


@dataclass
class ScalarProblem:
    mesh: Mesh
    sigma: np.ndarray
    bc_nodes: np.ndarray
    bc_values: np.ndarray


def cube_elastic(n: int = 20, jitter: float = 0.1, seed: int = 1234, E: float = 1.0, nu: float = 0.3,
                 n_spheres: int = 0, contrast: float = 1.0, sphere_seed: int = 7,
                 rmin: float = 0.02, rmax: float = 0.06) -> ElasticProblem:
    """Elastic cube: u = 0 on z = 0 (all three components), traction (0, 0, -1)
    on the z = 1 faces; optional spherical inclusions with E * contrast."""
    mesh = kuhn_cube(n, jitter=jitter, seed=seed)
    Es, nus = [E], [nu]
    if n_spheres > 0:
        centres, radii = random_spheres(n_spheres, rmin, rmax, sphere_seed)
        mark_spheres(mesh, centres, radii, 1)
        Es.append(E * contrast)
        nus.append(nu)
    bc = nodes_on_plane(mesh, 2, 0.0)
    faces, face_elem = boundary_faces_on_plane(mesh, 2, 1.0)
    traction = np.tile(np.array([0.0, 0.0, -1.0]), (faces.shape[0], 1))
    return ElasticProblem(
        mesh=mesh, E=np.array(Es), nu=np.array(nus), bc_nodes=bc,
        bc_mask=np.full(bc.size, 7, dtype=np.int32), bc_values=np.zeros((bc.size, 3)),
        faces=faces, face_elem=face_elem, traction=traction,
    )


def cube_scalar(n: int = 100, jitter: float = 0.0, seed: int = 1234, n_spheres: int = 200, contrast: float = 100.0,
                sphere_seed: int = 2024, rmin: float = 0.02, rmax: float = 0.06) -> ScalarProblem:
    """Electrostatics cube: permittivity 1, `contrast` inside spheres; potential 1
    on x = 0 and 0 on x = 1.  Dirichlet nodes are listed x = 0 face first, then
    x = 1 face, each ascending, as two boundary "types" would be read."""
    mesh = kuhn_cube(n, jitter=jitter, seed=seed)
    sig = [1.0]
    if n_spheres > 0:
        centres, radii = random_spheres(n_spheres, rmin, rmax, sphere_seed)
        mark_spheres(mesh, centres, radii, 1)
        sig.append(contrast)
    left = nodes_on_plane(mesh, 0, 0.0)
    right = nodes_on_plane(mesh, 0, 1.0)
    nodes = np.concatenate([left, right]).astype(np.int32)
    vals = np.concatenate([np.ones(left.size), np.zeros(right.size)])
    return ScalarProblem(mesh=mesh, sigma=np.array(sig), bc_nodes=nodes, bc_values=vals)


# ----------------------------------------------------------------------------------------------
# MsFEM macro cells, each with its own fine mesh
# ----------------------------------------------------------------------------------------------

@dataclass
class CellMeshes:
    """Concatenated per-cell fine meshes (cell-local tet node ids, as the
    reference's per-cell NVTR files hold them, MsFEM/MsFEM_Grid.h:4837)."""
    node_off: np.ndarray   # int64 [n_cells + 1]
    xyz: np.ndarray        # float64 [n_nodes, 3]
    tet_off: np.ndarray    # int64 [n_cells + 1]
    tets: np.ndarray       # int32 [n_tets, 4], cell-local
    mat: np.ndarray        # int32 [n_tets]
    box: np.ndarray        # float64 [n_cells, 6] (x0, x1, y0, y1, z0, z1)
    E: np.ndarray
    nu: np.ndarray
    m: np.ndarray          # int32 [n_cells] fine hexahedra per cell edge

    @property
    def n_cells(self) -> int:
        return int(self.box.shape[0])

    def cell(self, c: int):
        """(xyz, tets (local), mat, box) of cell c."""
        a, b = self.node_off[c], self.node_off[c + 1]
        s, t = self.tet_off[c], self.tet_off[c + 1]
        return self.xyz[a:b], self.tets[s:t], self.mat[s:t], self.box[c]


def msfem_cells(n_coarse: int = 16, m_choices=(8, 12, 16, 20), seed: int = 3, max_inclusions: int = 3,
                contrast: float = 50.0, nu: float = 0.3, semi=(0.15, 0.45), cells=None) -> CellMeshes:
    """n_coarse^3 macro cells on the unit cube; cell (i, j, k) (index i + n(j + n k)) is the box
    [i/n, (i+1)/n] x ..., meshed by kuhn_cube(m) with m drawn per cell from m_choices.  Each
    cell holds 1..max_inclusions axis-aligned ellipsoids (centres U(0,1)^3 and semi-axes
    U(semi) in cell units) whose tets (by centroid) take material 1 with E = contrast.
    `cells` restricts the batch to the listed cell indices (the draws stay those of the full grid)."""
    rng = np.random.default_rng(seed)
    n_all = n_coarse ** 3
    ms = rng.choice(np.asarray(m_choices), size=n_all)
    n_inc = rng.integers(1, max_inclusions + 1, size=n_all)
    cen = rng.uniform(0.0, 1.0, size=(n_all, max_inclusions, 3))
    ax = rng.uniform(semi[0], semi[1], size=(n_all, max_inclusions, 3))
    sel = np.arange(n_all) if cells is None else np.asarray(cells)
    h = 1.0 / n_coarse
    templ = {}
    for m in np.unique(ms[sel]):
        t = kuhn_cube(int(m))
        templ[int(m)] = (t.xyz, t.tets, tet_centroids(t))
    xyzs, tetss, mats, boxes, noff, toff = [], [], [], [], [0], [0]
    for c in sel:
        i, j, k = c % n_coarse, (c // n_coarse) % n_coarse, c // (n_coarse * n_coarse)
        lo = np.array([i, j, k], dtype=np.float64) * h
        uxyz, utets, ucen = templ[int(ms[c])]
        xyzs.append(lo + uxyz * h)
        inside = np.zeros(utets.shape[0], dtype=bool)
        for q in range(n_inc[c]):
            inside |= (((ucen - cen[c, q]) / ax[c, q]) ** 2).sum(axis=1) < 1.0
        tetss.append(utets)
        mats.append(inside.astype(np.int32))
        boxes.append([lo[0], lo[0] + h, lo[1], lo[1] + h, lo[2], lo[2] + h])
        noff.append(noff[-1] + uxyz.shape[0])
        toff.append(toff[-1] + utets.shape[0])
    return CellMeshes(node_off=np.array(noff, dtype=np.int64), xyz=np.concatenate(xyzs),
                      tet_off=np.array(toff, dtype=np.int64), tets=np.concatenate(tetss).astype(np.int32),
                      mat=np.concatenate(mats), box=np.array(boxes), E=np.array([1.0, contrast]),
                      nu=np.array([nu, nu]), m=ms[sel].astype(np.int32))


def subset_cells(cm: CellMeshes, idx) -> CellMeshes:
    """The cells `idx` of cm (in that order) as their own CellMeshes."""
    idx = np.asarray(idx, dtype=np.int64)
    nn = cm.node_off[idx + 1] - cm.node_off[idx]
    nt = cm.tet_off[idx + 1] - cm.tet_off[idx]
    node_rows = np.concatenate([np.arange(cm.node_off[c], cm.node_off[c + 1]) for c in idx]) if idx.size else np.zeros(0, np.int64)
    tet_rows = np.concatenate([np.arange(cm.tet_off[c], cm.tet_off[c + 1]) for c in idx]) if idx.size else np.zeros(0, np.int64)
    return CellMeshes(node_off=np.concatenate([[0], np.cumsum(nn)]).astype(np.int64), xyz=cm.xyz[node_rows],
                      tet_off=np.concatenate([[0], np.cumsum(nt)]).astype(np.int64), tets=cm.tets[tet_rows],
                      mat=cm.mat[tet_rows], box=cm.box[idx], E=cm.E, nu=cm.nu, m=cm.m[idx])


def sphere_cells(n_cells: int, seed: int = 0, m: int = 8, density: float = 0.58, rmin: float = 0.24,
                 rmax: float = 0.56, contrast: float = 100.0, nu: float = 0.3, h: float = 1.0 / 16.0) -> CellMeshes:
    """n_cells independent macro cells of kuhn_cube(m) (edge h, laid out along x) cut from a random
    field of spherical inclusions like the elasticity workload's (2000 spheres of radius
    U(0.015, 0.035) in the unit cube cut into 16^3 cells: radii U(0.24, 0.56) in cell units, about
    13 % inclusion volume): sphere centres with `density` per cell volume, uniform over the cell
    grown by rmax on every side so that spheres of neighbouring cells cut in; no two spheres of a
    cell overlap (rejection in draw order, which favours small radii, as the workload's own
    placement does).  Tets whose centroid lies in a sphere take material 1
    (E = contrast, nu)."""
    rng = np.random.default_rng(seed)
    t = kuhn_cube(m)
    cen = tet_centroids(t)
    side = 1.0 + 2.0 * rmax
    xyzs, mats, boxes = [], [], []
    for c in range(n_cells):
        k = rng.poisson(density * side ** 3)
        cs, rs = [], []
        for _ in range(k):
            for _try in range(50):
                p = rng.uniform(-rmax, 1.0 + rmax, size=3)
                r = rng.uniform(rmin, rmax)
                if all(np.linalg.norm(p - q) >= r + s for q, s in zip(cs, rs)):
                    cs.append(p)
                    rs.append(r)
                    break
        inside = np.zeros(cen.shape[0], dtype=bool)
        for p, r in zip(cs, rs):
            inside |= ((cen - p) ** 2).sum(axis=1) < r * r
        lo = np.array([c * h, 0.0, 0.0])
        xyzs.append(lo + t.xyz * h)
        mats.append(inside.astype(np.int32))
        boxes.append([lo[0], lo[0] + h, 0.0, h, 0.0, h])
    nn, nt = t.xyz.shape[0], t.tets.shape[0]
    return CellMeshes(node_off=np.arange(n_cells + 1, dtype=np.int64) * nn, xyz=np.concatenate(xyzs),
                      tet_off=np.arange(n_cells + 1, dtype=np.int64) * nt,
                      tets=np.tile(t.tets, (n_cells, 1)).astype(np.int32), mat=np.concatenate(mats),
                      box=np.array(boxes), E=np.array([1.0, contrast]), nu=np.array([nu, nu]),
                      m=np.full(n_cells, m, dtype=np.int32))


@dataclass
class CubeCells:
    """A structured cube mesh (kuhn_cube(n)) cut into nc^3 macro cells of H = n/nc hexahedra
    per edge, each with its own copy of the fine mesh (cell-local numbering)."""
    cells: CellMeshes
    cell_node_global: np.ndarray   # int32 [cells' nodes]: fine node of each cell node
    cell_vertex: np.ndarray        # int32 [n_cells, 8]: coarse vertex of each cell corner
    cell_color: np.ndarray         # int32 [n_cells]: parity colour, cells of a colour share no vertex
    n_coarse_vertices: int


def cube_cells(mesh: Mesh, E, nu, H: int) -> CubeCells:
    """Cells of H^3 hexahedra over kuhn_cube(n) (n % H == 0); each cell keeps the fine mesh's own
    tetrahedra (same node order) renumbered cell-locally, so the cells' element blocks are the
    fine problem's element blocks."""
    n = mesh.n
    if n % H:
        raise ValueError("n must be a multiple of H")
    nc = n // H
    i = np.arange(H + 1)
    lk, lj, li = np.meshgrid(i, i, i, indexing="ij")
    li, lj, lk = li.ravel(), lj.ravel(), lk.ravel()          # local node (i, j, k), id li + (H+1)(lj + (H+1)lk)
    hx = np.arange(H)
    hk, hj, hi = np.meshgrid(hx, hx, hx, indexing="ij")
    hi, hj, hk = hi.ravel(), hj.ravel(), hk.ravel()          # local hexahedra
    xyzs, tets, mats, boxes, cng, cvert, color = [], [], [], [], [], [], []
    noff, toff = [0], [0]
    for c in range(nc ** 3):
        ci, cj, ck = c % nc, (c // nc) % nc, c // (nc * nc)
        g = node_id(n, ci * H + li, cj * H + lj, ck * H + lk)
        hexes = (ci * H + hi) + n * ((cj * H + hj) + n * (ck * H + hk))
        te = (hexes[:, None] * 6 + np.arange(6)[None, :]).ravel()
        loc = np.full(mesh.n_nodes, -1, dtype=np.int64)
        loc[g] = np.arange(g.size)
        xyzs.append(mesh.xyz[g])
        tets.append(loc[mesh.tets[te]])
        mats.append(mesh.mat[te])
        h = 1.0 / nc
        boxes.append([ci * h, (ci + 1) * h, cj * h, (cj + 1) * h, ck * h, (ck + 1) * h])
        cng.append(g)
        cvert.append([(ci + (v & 1)) + (nc + 1) * ((cj + ((v >> 1) & 1)) + (nc + 1) * (ck + ((v >> 2) & 1)))
                      for v in range(8)])
        color.append((ci & 1) | ((cj & 1) << 1) | ((ck & 1) << 2))
        noff.append(noff[-1] + g.size)
        toff.append(toff[-1] + te.size)
    cm = CellMeshes(node_off=np.array(noff, dtype=np.int64), xyz=np.concatenate(xyzs),
                    tet_off=np.array(toff, dtype=np.int64), tets=np.concatenate(tets).astype(np.int32),
                    mat=np.concatenate(mats).astype(np.int32), box=np.array(boxes), E=np.asarray(E, float),
                    nu=np.asarray(nu, float), m=np.full(nc ** 3, H, dtype=np.int32))
    return CubeCells(cells=cm, cell_node_global=np.concatenate(cng).astype(np.int32),
                     cell_vertex=np.array(cvert, dtype=np.int32), cell_color=np.array(color, dtype=np.int32),
                     n_coarse_vertices=(nc + 1) ** 3)


# ------------------------------------------------------------------ the benchmark workloads

def heterogeneous_elasticity(n: int = 128):
    """The 128^3 heterogeneous elasticity workload (and its smaller sizes): n^3 hexahedra of six Kuhn
    tetrahedra on the unit cube, 2000 seeded non-overlapping spheres (radii U(0.015, 0.035),
    sphere seed 4096) with E contrast 1:100, nu 0.3, u = 0 on z = 0, traction (0, 0, -1) on z = 1.
    The spheres do not depend on n."""
    return cube_elastic(n=n, jitter=0.0, n_spheres=2000, contrast=100.0, rmin=0.015, rmax=0.035, sphere_seed=4096)


def electrostatics(n: int = 100):
    """The 100^3 electrostatics workload (and its smaller sizes): permittivity 1, and 100 inside 200
    seeded non-overlapping spheres (radii U(0.02, 0.06), sphere seed 2024); potential 1 on x = 0 and
    0 on x = 1."""
    return cube_scalar(n=n, n_spheres=200, contrast=100.0, rmin=0.02, rmax=0.06, sphere_seed=2024)
