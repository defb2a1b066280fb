"""The MsFEM Order1 restatement (oracle/cells.py, oracle/msfem.py) against the reference's own
Order1 construction and driver run here (oracle/_ref/order2_ref --order1:
MsFEM_forElasticDeformation_OrderBF1_forPoly on Grid_forMech_Poly_Order1, MsFEM/MsFEM.h:571-1062,
on a macro mesh and cell directories written by meshio)."""
import os
import types

import numpy as np
import pytest

from oracle import cells as oc
from oracle import msfem as om
from oracle import order2 as o2

pytestmark = pytest.mark.skipif(not os.path.exists(o2.ORDER2_REF),
                                reason="oracle/_ref/order2_ref not built (make -C oracle ref)")


@pytest.fixture(scope="module")
def order1_run(tmp_path_factory):
    vxyz, cv, cm = o2.graded_cells(2, 4, 0.5)
    bot = np.nonzero(np.abs(vxyz[:, 2]) < 1e-12)[0]
    top = np.nonzero(np.abs(vxyz[:, 2] - 1) < 1e-12)[0]
    groups = [(bot, (0.0, 0.0, 0.0), (1, 1, 1)), (top, (0.01, -0.02, 0.05), (1, 1, 1))]
    R = o2.run_reference(str(tmp_path_factory.mktemp("order1")), vxyz, cv, cm, matrices=False, groups=groups,
                         min_residual=1e-13, order1=True)
    return vxyz, cv, cm, groups, R


def test_order1_bases_match_reference_construction(order1_run):
    """8 graded cells with inclusions (E 1:10): with material 0 on the face and edge problems (the
    reference's Salome face meshes carry no materials) the restated bases equal the reference's
    within 1e-11; with the tetrahedra's materials on the faces they do not."""
    vxyz, cv, cm, groups, R = order1_run
    worst_zero, worst_cells = 0.0, 0.0
    for c in range(cm.n_cells):
        xyz, tets, mat, box = cm.cell(c)
        ref = R["bases"][c]
        z = oc.order1_bases(xyz, tets, mat, box, cm.E, cm.nu, face_material="zero")
        worst_zero = max(worst_zero, np.abs(z - ref).max())
        if mat.any():
            w = oc.order1_bases(xyz, tets, mat, box, cm.E, cm.nu, face_material="cells")
            worst_cells = max(worst_cells, np.abs(w - ref).max())
    assert worst_zero < 1e-11
    assert worst_cells > 1e-3


def test_order1_driver_matches_reference(order1_run):
    """The whole Order1 driver (Dirichlet groups on z = 0 and z = 1): the restated driver on the
    restated bases gives the reference's macro solution within 1e-9."""
    vxyz, cv, cm, groups, R = order1_run
    bases = np.concatenate([oc.order1_bases(*cm.cell(c)[:3], cm.cell(c)[3], cm.E, cm.nu, face_material="zero")
                            for c in range(cm.n_cells)])
    cc = types.SimpleNamespace(cells=cm, cell_vertex=cv, n_coarse_vertices=vxyz.shape[0])
    fv = np.concatenate([g[0] for g in groups])
    vals = np.concatenate([np.tile(g[1], (len(g[0]), 1)) for g in groups])
    U, _, _, _ = om.driver(cc, bases, fv, vals, [], [], cm.E[0], cm.nu[0])
    ref = R["solution"]
    assert np.linalg.norm(U - ref) <= 1e-9 * np.linalg.norm(ref)
