"""The cracked-conduction restatement (multiscalefemsolver3d_b200/xfem.py, oracle/xfem.py) against
exact answers: side volumes of a clipped tetrahedron, a crack through the whole cube (the two
halves decouple: T = 1 below it, 0 above, exactly in the enriched space), and no crack at all
(the plain P1 assembly)."""
import numpy as np
import pytest

from multiscalefemsolver3d_b200 import meshgen, xfem
from oracle import xfem as ox


def test_side_fraction_exact_cases():
    # the reference tetrahedron (0,0,0),(1,0,0),(0,1,0),(0,0,1) cut by x + y + z = t: volume t^3
    P = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1.0]])
    for t in (0.1, 0.5, 0.9):
        d = t - P.sum(axis=1)                     # >= 0 on the corner side
        assert xfem.side_fraction(d) == pytest.approx(t ** 3, rel=1e-14)
        assert xfem.side_fraction(-d) == pytest.approx(1 - t ** 3, rel=1e-14)
    # a 2-2 split by x = 1/2 on the same tet: the slab x >= 1/2 has volume (1/2)^3 of the tet
    d = P[:, 0] - 0.5
    assert xfem.side_fraction(d) == pytest.approx(0.125, rel=1e-14)
    # symmetric 2-2 values give one half; ties and zeros stay finite
    assert xfem.side_fraction(np.array([1.0, 1.0, -1.0, -1.0])) == pytest.approx(0.5, rel=1e-15)
    rng = np.random.default_rng(0)
    for _ in range(200):
        d = rng.normal(size=4)
        f = xfem.side_fraction(d)
        assert 0.0 <= f <= 1.0 and f + xfem.side_fraction(-d) == pytest.approx(1.0, abs=1e-12)
    # Monte Carlo against the definition on a 2-2 case
    d = np.array([0.7, 0.2, -0.4, -0.9])
    lam = rng.dirichlet(np.ones(4), size=400000)
    assert xfem.side_fraction(d) == pytest.approx(float(((lam @ d) >= 0).mean()), abs=3e-3)


def test_full_crack_decouples_the_halves():
    mesh = meshgen.kuhn_cube(6, jitter=0.05, seed=1)
    cr = xfem.Cracks(centre=np.array([[0.5, 0.5, 0.53]]), normal=np.array([[0.0, 0.0, 1.0]]), radius=np.array([10.0]))
    enr = xfem.enrich(mesh.xyz, mesh.tets, cr)
    assert enr.n_enriched > 0
    A = ox.assemble(mesh.xyz, mesh.tets, np.ones(mesh.n_tets), cr, enr)
    assert abs(A - A.T).max() <= 1e-14 * abs(A).max()
    lo = meshgen.nodes_on_plane(mesh, 2, 0.0)
    hi = meshgen.nodes_on_plane(mesh, 2, 1.0)
    x = ox.solve_dirichlet(A, np.concatenate([lo, hi]), np.concatenate([np.ones(lo.size), np.zeros(hi.size)]))
    # temperature at each vertex side: standard value, and across the crack inside cut tets
    T = x[:mesh.n_nodes]
    below = mesh.xyz[:, 2] < 0.53
    np.testing.assert_allclose(T[below], 1.0, atol=1e-10)
    np.testing.assert_allclose(T[~below], 0.0, atol=1e-10)


def test_no_crack_is_the_plain_assembly():
    mesh = meshgen.kuhn_cube(4, jitter=0.1, seed=2)
    cr = xfem.Cracks(centre=np.array([[5.0, 5.0, 5.0]]), normal=np.array([[0.0, 0.0, 1.0]]), radius=np.array([0.1]))
    enr = xfem.enrich(mesh.xyz, mesh.tets, cr)
    assert enr.n_enriched == 0 and enr.n_dofs == mesh.n_nodes
    sig = np.random.default_rng(3).uniform(1, 5, mesh.n_tets)
    A = ox.assemble(mesh.xyz, mesh.tets, sig, cr, enr)
    g, V = ox._grads(mesh.xyz[mesh.tets])
    Kd = np.einsum("eid,eid->e", g, g) * sig * V          # trace of each element matrix
    assert A.diagonal().sum() == pytest.approx(Kd.sum(), rel=1e-13)
    np.testing.assert_allclose(A @ np.ones(mesh.n_nodes), 0.0, atol=1e-12 * abs(A).max())


def test_random_cracks_workload_statistics():
    mesh, cr, nodes, vals = xfem.cube_cracked(n=16, n_cracks=10, seed=5)
    enr = xfem.enrich(mesh.xyz, mesh.tets, cr)
    assert cr.radius.min() >= 0.03 and cr.radius.max() <= 0.1
    assert enr.n_enriched > 0 and (enr.crack_of_tet >= 0).sum() > 0
    # every enriched DOF belongs to exactly one (crack, node) pair and appears in a cut tet
    used = np.unique(enr.enr_dof[enr.enr_dof >= 0])
    np.testing.assert_array_equal(used, np.arange(mesh.n_nodes, enr.n_dofs))


def test_side_fractions_closed_form_against_clipping():
    """The product's closed-form side fractions (host, and the device copy in csrc/xfem.cu) against
    the oracle's geometric clipping, over random tetrahedra and planes (all sign patterns)."""
    rng = np.random.default_rng(7)
    for _ in range(2000):
        P = rng.normal(size=(4, 3))
        d = rng.normal(size=4)
        assert xfem.side_fraction(d) == pytest.approx(ox.clip_fraction(P, d), abs=1e-12)


def test_enrichment_matches_loop_restatement():
    """Cut detection and enriched numbering of the product (vectorised, z-slab bucketing) against
    the oracle's tetrahedron-by-tetrahedron loops, on a jittered mesh with overlapping cracks."""
    mesh = meshgen.kuhn_cube(10, jitter=0.1, seed=4)
    cr = xfem.random_cracks(25, 0.05, 0.3, seed=2)
    a = xfem.enrich(mesh.xyz, mesh.tets, cr)
    b = ox.enrich(mesh.xyz, mesh.tets, cr)
    assert a.n_enriched > 0 and a.n_dofs == b.n_dofs and a.n_enriched == b.n_enriched
    np.testing.assert_array_equal(a.crack_of_tet, b.crack_of_tet)
    np.testing.assert_array_equal(a.enr_dof, b.enr_dof)
