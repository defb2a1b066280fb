"""Generates the reference solutions of the two benchmark workloads at reduced size, the largest
each CPU restatement or the reference itself solves in minutes here (run once; the fixtures are
committed so the GPU tests and bench.py need neither the reference nor a long CPU solve):

    python tests/golden/make_workload_solutions.py [--elastic] [--scalar]

  elastic_c4_n32.npz  meshgen.heterogeneous_elasticity(32) (107,811 DOF: 2000 spheres, E 1:100): the
                      system assembled by the C restatement (oracle/femoracle.c, pinned to the
                      reference's assembly) solved by sparse LU in FP64 -- the reference's own
                      solvers do not reach 1e-8 on this indefinite system; about 5 minutes
  scalar_c2_n60.npz   meshgen.electrostatics(60) (226,981 DOF): the reference's own
                      FEM::FEM_forBaseEliptic (stiffness-only, FEM/FEM.h:398-717, SSOR-PCG restart
                      loop to MIN_RESIDUAL 1e-10) run here through oracle/_ref/libfemref.so
Each stores the solution and a coordinate checksum of the generated mesh.
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


def elastic(n=32):
    import scipy.sparse.linalg as spl
    p = meshgen.heterogeneous_elasticity(n)
    A = oracle.port().elastic_system(p, stage=1)
    t0 = time.perf_counter()
    x = spl.spsolve(A.to_scipy().tocsc(), A.F)
    t = time.perf_counter() - t0
    rel = float(np.linalg.norm(A.F - A.to_scipy() @ x) / np.linalg.norm(A.F))
    np.savez_compressed(os.path.join(HERE, f"elastic_c4_n{n}.npz"), n=n, xyz_sum=p.mesh.xyz.sum(), x=x,
                        rel_residual=rel, seconds=t)
    print(f"elastic n={n}: {A.n} DOF, sparse LU {t:.1f} s, relative residual {rel:.2e}")


def scalar(n=60):
    p = meshgen.electrostatics(n)
    x, wall = oracle.ref().scalar_driver(p, min_residual=1e-10, nthreads=os.cpu_count() or 1)
    A = oracle.port().scalar_system(p, stage=1)
    rel = float(np.linalg.norm(A.F - A.to_scipy() @ x) / np.linalg.norm(A.F))
    np.savez_compressed(os.path.join(HERE, f"scalar_c2_n{n}.npz"), n=n, xyz_sum=p.mesh.xyz.sum(), x=x,
                        rel_residual=rel, seconds=wall)
    print(f"scalar n={n}: {x.size} DOF, reference driver {wall:.1f} s, relative residual {rel:.2e}")


if __name__ == "__main__":
    which = [a for a in sys.argv[1:] if a.startswith("--")]
    if not which or "--scalar" in which:
        scalar()
    if not which or "--elastic" in which:
        elastic()
