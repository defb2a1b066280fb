"""A short, fixed GPU case for profilers (ncu): the electrostatics workload at
size n^3, one assembled system, optionally one FP32-IR solve to 1e-8, then
2 + 3 warm-up SpMV products in FP32 and in FP64 (msfem_bench_spmv).

    python -m multiscalefemsolver3d_b200.profile_case --n 120 --solve

Kernel launch order (for ncu -k/-s/-c): portrait and assembly kernels, the
Dirichlet kernels, the solve (if --solve), then k_spmv<float> x5, then
k_spmv<double> x5.
"""
from __future__ import annotations

import argparse
import json


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=120)
    ap.add_argument("--solve", action="store_true")
    ap.add_argument("--elastic", action="store_true", help="elasticity cube instead of electrostatics")
    a = ap.parse_args()
    from . import fem, meshgen
    if a.elastic:
        p = meshgen.cube_elastic(n=a.n, n_spheres=200, contrast=100.0, rmin=0.02, rmax=0.06)
        S = fem.System(fem.ELASTIC, p.mesh.xyz, p.mesh.tets, p.mesh.mat)
        S.add_traction(p.faces, p.traction)
        S.assemble_elastic(p.E, p.nu)
        dofs = (3 * p.bc_nodes[:, None] + [0, 1, 2]).ravel().astype("int32")
        S.apply_dirichlet(dofs, p.bc_values.ravel(), fem.ROW_AND_COLUMN)
    else:
        p = meshgen.cube_scalar(n=a.n, n_spheres=200, contrast=100.0, rmin=0.02, rmax=0.06, sphere_seed=2024)
        S = fem.System(fem.SCALAR, p.mesh.xyz, p.mesh.tets, p.mesh.mat)
        S.assemble_scalar(p.sigma)
        S.apply_dirichlet(p.bc_nodes, p.bc_values, fem.ROW_AND_COLUMN)
        S.copy_f_to_x()
    out = {"n": a.n, "rows": S.n_rows, "nnz": S.nnz}
    if a.solve:
        rel, it, rc = S.solve(fem.PCG_JACOBI, fem.FP32_IR, tol=1e-8, maxiter=200000)
        out.update(rel=rel, iterations=it, rc=rc, stats=S.stats())
    ms32, b32 = S.bench_spmv(fem.FP32_IR, reps=2)
    ms64, b64 = S.bench_spmv(fem.FP64, reps=2)
    out.update(spmv32_ms=ms32, spmv32_bytes=b32, spmv64_ms=ms64, spmv64_bytes=b64)
    S.close()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
