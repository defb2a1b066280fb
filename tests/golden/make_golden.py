"""Generates the golden fixtures in this directory from the reference itself
(oracle/_ref/libfemref.so, compiled from the reference's sources by
oracle/Makefile).  Run once where the reference is available:

    python tests/golden/make_golden.py

Fixtures (all inputs are regenerated from the stored mesh parameters by
multiscalefemsolver3d_b200.meshgen; a coordinate checksum guards against drift):
  unit_tets.npz    element matrices (FEM_Grid.h:2125-2192, :103-152) of 4 tetrahedra
  elastic_n3.npz   FEM_forElasticDeformation system after BCs (FEM.h:1286-1813), 3^3 cube,
                   and the reference CG (MSG) solution to 1e-13
  scalar_n6.npz    stiffness-only FEM_forBaseEliptic system after BCs (FEM.h:398-635), 6^3 cube
                   with 3 spheres, the reference CG solution and the driver's own output
  c1_elastic.npz   the 20^3 elasticity workload (27,783 DOF): matrix checksums, the reference CG
                   solution to 1e-12 on the reference-assembled system, and the driver's output
  msfem_order1.npz the reference's whole MsFEM Order1 run (oracle/_ref/order2_ref --order1) on
                   oracle.order2.graded_cells(2, 4, 0.5): the bases of cells 0 and 7 and the
                   driver's macro solution for u = 0 on z = 0, u = (0.01, -0.02, 0.05) on z = 1
  msfem_order2.npz the reference's Order2 construction on graded_cells(1, 4, 0.5): the 27 bases
                   and the macro element matrix; and its whole Order2 driver on graded_cells(2, 4,
                   0.5) with the same Dirichlet groups: the macro solution
Only the MsFEM fixtures:  python tests/golden/make_golden.py --msfem
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from multiscalefemsolver3d_b200 import meshgen  # noqa: E402

UNIT = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], dtype=float)


def main():
    R = oracle.ref()
    rng = np.random.default_rng(42)
    tets = [UNIT] + [UNIT * rng.uniform(0.3, 2.0) + rng.normal(0, 0.1, (4, 3)) for _ in range(3)]
    mats = [(1.0, 0.3), (30.0, 0.25), (2.5, 0.45), (100.0, 0.1)]
    np.savez_compressed(os.path.join(HERE, "unit_tets.npz"), xyz=np.array(tets), E=np.array([m[0] for m in mats]),
                        nu=np.array([m[1] for m in mats]),
                        K_elastic=np.array([R.elastic_local(t, *m) for t, m in zip(tets, mats)]),
                        K_scalar=np.array([R.scalar_local(t, m[0]) for t, m in zip(tets, mats)]))

    p = meshgen.cube_elastic(n=3)
    A, _ = R.elastic_system(p, stage=1)
    x, res, _ = R.cssd_solve(0, A, tol=1e-13)
    np.savez_compressed(os.path.join(HERE, "elastic_n3.npz"), n=3, jitter=0.1, seed=1234,
                        xyz_sum=p.mesh.xyz.sum(), row_ptr=A.row_ptr, col=A.col, val=A.val, F=A.F, X=A.X,
                        x_cg=x, cg_residual=res)

    p = meshgen.cube_scalar(n=6, n_spheres=3, rmin=0.1, rmax=0.2)
    A, _ = R.scalar_system(p, stage=1)
    x, res, _ = R.cssd_solve(0, A, tol=1e-13)
    xd, _ = R.scalar_driver(p, min_residual=1e-10)
    np.savez_compressed(os.path.join(HERE, "scalar_n6.npz"), n=6, spheres=3, rmin=0.1, rmax=0.2,
                        mat=p.mesh.mat, xyz_sum=p.mesh.xyz.sum(), row_ptr=A.row_ptr, col=A.col, val=A.val,
                        F=A.F, X=A.X, x_cg=x, cg_residual=res, x_driver=xd)

    p = meshgen.cube_elastic(n=20)
    t0 = time.time()
    A, _ = R.elastic_system(p, stage=1, nthreads=os.cpu_count())
    x, res, wall = R.cssd_solve(0, A, tol=1e-12, nthreads=os.cpu_count())
    xd, wd = R.elastic_driver(p, min_residual=1e-10, nthreads=os.cpu_count())
    np.savez_compressed(os.path.join(HERE, "c1_elastic.npz"), n=20, jitter=0.1, seed=1234,
                        xyz_sum=p.mesh.xyz.sum(), nnz=A.row_ptr[-1], col_sum=int(A.col.astype(np.int64).sum()),
                        val_abs_sum=np.abs(A.val).sum(), val_fro=np.linalg.norm(A.val), F=A.F, x_cg=x,
                        cg_residual=res, x_driver=xd, driver_wall_s=wd)
    print(f"c1: cg residual {res:.2e} ({wall:.1f} s), driver {wd:.1f} s, total {time.time() - t0:.1f} s")


def msfem():
    import tempfile

    from oracle import order2 as o2

    def groups_of(vxyz):
        bot = np.nonzero(np.abs(vxyz[:, 2]) < 1e-12)[0]
        top = np.nonzero(np.abs(vxyz[:, 2] - 1) < 1e-12)[0]
        return [(bot, (0.0, 0.0, 0.0), (1, 1, 1)), (top, (0.01, -0.02, 0.05), (1, 1, 1))]

    vxyz, cv, cm = o2.graded_cells(2, 4, 0.5)
    R1 = o2.run_reference(tempfile.mkdtemp(), vxyz, cv, cm, matrices=False, groups=groups_of(vxyz),
                          min_residual=1e-13, order1=True)
    np.savez_compressed(os.path.join(HERE, "msfem_order1.npz"), xyz_sum=cm.xyz.sum(), bases_0=R1["bases"][0],
                        bases_7=R1["bases"][7], solution=R1["solution"])
    vxyz1, cv1, cm1 = o2.graded_cells(1, 4, 0.5)
    R2 = o2.run_reference(tempfile.mkdtemp(), vxyz1, cv1, cm1, matrices=True)
    R3 = o2.run_reference(tempfile.mkdtemp(), vxyz, cv, cm, matrices=False, groups=groups_of(vxyz),
                          min_residual=1e-13)
    np.savez_compressed(os.path.join(HERE, "msfem_order2.npz"), xyz_sum_1=cm1.xyz.sum(), bases=R2["bases"][0],
                        K=R2["K"][0], cell_dofs=R3["cell_dofs"], xyz_sum_2=cm.xyz.sum(), solution=R3["solution"])


if __name__ == "__main__":
    if "--msfem" in sys.argv:
        msfem()
    else:
        main()
        msfem()
