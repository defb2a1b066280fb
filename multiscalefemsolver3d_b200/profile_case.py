"""A short, fixed GPU case for profilers (ncu): the electrostatics workload at
size n^3, one assembled system, optionally one FP32-IR solve to 1e-8, then
2 + 3 warm-up SpMV products in FP32 and in FP64 (msfem_bench_spmv).

    python -m multiscalefemsolver3d_b200.profile_case --n 120 --solve

Kernel launch order (for ncu -k/-s/-c): portrait and assembly kernels, the
Dirichlet kernels, the solve (if --solve), then k_spmv<float> x5, then
k_spmv<double> x5.

    python -m multiscalefemsolver3d_b200.profile_case --twolevel --n 64 [--maxiter K]

runs the two-level elasticity solve of the 128^3 workload (meshgen.heterogeneous_elasticity) at
n^3 (n/8 macro cells per axis): both assemblies, Dirichlet, the exact cell bases, coarse setup,
the multiplicative cycle and FP64 MINRES to 1e-8 (or K iterations: every iteration launches the
same kernels, so a launch list of a few hundred iterations shows the solve's mix).

    python -m multiscalefemsolver3d_b200.profile_case --cells 8

runs the batched Order1 cell bases of n^3 macro cells of the 16^3-cell workload's kind (per-cell
resolution from {8, 12, 16, 20}, ellipsoidal inclusions E 1:50): edges, faces, volumes.

    python -m multiscalefemsolver3d_b200.profile_case --order2 8

runs the batched Order2 cell bases (27 per cell) of the same n^3 cells, after their Order1 bases
for comparison: face problems (R = 8), then the four volume passes (R = 8 each).

    python -m multiscalefemsolver3d_b200.profile_case --net 512

predicts the bases of 512 sphere cells with the learned coarse space on each tensor-core path of
layers 1-3 in turn (0: mma.sync k_conv32, 1: k_conv32_tc, 2: k_conv32_tt, 3: k_conv32_ws), five
predictions per path, and prints the device time of each path.
"""
from __future__ import annotations

import argparse
import json


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=120)
    ap.add_argument("--solve", action="store_true")
    ap.add_argument("--elastic", action="store_true", help="elasticity cube instead of electrostatics")
    ap.add_argument("--twolevel", action="store_true", help="two-level elasticity solve at n^3")
    ap.add_argument("--cells", type=int, default=0, help="batched cell bases of cells^3 macro cells")
    ap.add_argument("--net", type=int, default=0, help="network forward passes over this many cells")
    ap.add_argument("--order2", type=int, default=0, help="batched Order2 bases of order2^3 macro cells")
    ap.add_argument("--maxiter", type=int, default=400000, help="two-level: MINRES iteration limit")
    ap.add_argument("--matrix-free", action="store_true", help="two-level: matrix-free operators on the Kuhn grid")
    ap.add_argument("--smoother-reps", type=int, default=0, help="two-level: time this many smoothing steps first")
    ap.add_argument("--sweep-smoother", action="store_true",
                    help="two-level at n^3: every Chebyshev degree of --degrees x ratio of --ratios")
    ap.add_argument("--degrees", default="2,3,4,5")
    ap.add_argument("--ratios", default="10,30,100")
    a = ap.parse_args()
    from . import fem, meshgen
    if a.order2:
        return order2_case(a.order2)
    if a.net:
        return net_case(a.net)
    if a.cells:
        return cells_case(a.cells)
    if a.twolevel:
        return twolevel_case(a.n, a.maxiter, a.matrix_free, a.smoother_reps)
    if a.sweep_smoother:
        return smoother_sweep(a.n, [int(v) for v in a.degrees.split(",")], [float(v) for v in a.ratios.split(",")],
                              a.maxiter)
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


def cells_case(nc):
    from . import meshgen
    from .cells import FP32_IR, Cells
    cm = meshgen.msfem_cells(n_coarse=nc, m_choices=(8, 12, 16, 20), seed=3, max_inclusions=3, contrast=50.0)
    C = Cells(cm)
    rc = C.build_bases(FP32_IR, 1e-8)
    r = C.report()
    print(json.dumps({"cells": cm.n_cells, "nodes": C.n_nodes, "rc": rc, "ms": r["ms"]}, default=str))
    C.close()


def order2_case(nc):
    import time

    import numpy as np

    from . import meshgen
    from .cells import FP32_IR, Cells
    cm = meshgen.msfem_cells(n_coarse=nc, m_choices=(8, 12, 16, 20), seed=3, max_inclusions=3, contrast=50.0)
    cv = np.array([[(c % nc + (b & 1)) + (nc + 1) * ((c // nc % nc + (b >> 1 & 1)) + (nc + 1) * (c // nc ** 2 + (b >> 2 & 1)))
                    for b in range(8)] for c in range(nc ** 3)], dtype=np.int32)
    C = Cells(cm)
    t0 = time.perf_counter()
    rc1 = C.build_bases(FP32_IR, 1e-8)
    t1 = time.perf_counter()
    rc2 = C.build_order2(cv, FP32_IR, 1e-8)
    t2 = time.perf_counter()
    C.build_order2(cv, FP32_IR, 1e-8)
    t3 = time.perf_counter()
    print(json.dumps({"cells": cm.n_cells, "nodes": C.n_nodes, "rc_order1": rc1, "rc_order2": rc2,
                      "s_order1_first": t1 - t0, "s_order2_first": t2 - t1, "s_order2_again": t3 - t2}))
    C.close()


def smoother_sweep(n, degrees, ratios, maxiter=400000):
    """The two-level solve of the heterogeneous elasticity case at n^3 (exact MsFEM bases, the
    cells' own face materials, matrix-free operators) for every Chebyshev degree x spectrum ratio:
    one JSON line each with iterations, solve time and ms per iteration."""
    import numpy as np

    from . import fem, meshgen
    from .cells import FP32_IR, FP64, Cells
    from .twolevel import TwoLevel
    p = meshgen.heterogeneous_elasticity(n)
    m = p.mesh
    dofs = (3 * p.bc_nodes[:, None] + np.arange(3)).ravel().astype(np.int32)
    zval = np.zeros(dofs.size)
    S = fem.System(fem.ELASTIC, m.xyz, m.tets, m.mat)
    S.add_traction(p.faces, p.traction)
    S.assemble_elastic(p.E, p.nu)
    S.apply_dirichlet(dofs, zval, fem.ROW_AND_COLUMN)
    K = fem.System(fem.ELASTIC, m.xyz, m.tets, m.mat)
    K.assemble_elastic_textbook(p.E, p.nu)
    K.apply_dirichlet(dofs, zval, fem.ROW_AND_COLUMN)
    S.set_kuhn_grid(n)
    K.set_kuhn_grid(n)
    cc = meshgen.cube_cells(m, p.E, p.nu, 8)
    C = Cells(cc.cells)
    C.set_face_material("cells")
    C.build_bases(FP32_IR, 1e-8)
    for deg in degrees:
        for ratio in ratios:
            T = TwoLevel(S, C, cc, dofs)
            T.set_smoother(K, degree=deg, ratio=ratio, matrix_free=True)
            T.set_matrix_free(True)
            S.set_x(np.zeros(S.n_rows))
            rel, it, out, rc = T.solve(tol=1e-8, maxiter=maxiter, precision=FP64)
            ms = S.stats()["ms_solve"]
            print(json.dumps({"n": n, "degree": deg, "ratio": ratio, "rc": rc, "rel": rel, "iterations": it,
                              "ms_solve": ms, "ms_per_iteration": ms / max(1, it),
                              "widened": T.stats()["widened"]}), flush=True)
            T.close()
    C.close()
    K.close()
    S.close()


def twolevel_case(n, maxiter=400000, matrix_free=False, smoother_reps=0):
    import numpy as np

    from . import fem, meshgen
    from .cells import FP32_IR, FP64, Cells
    from .twolevel import TwoLevel
    p = meshgen.heterogeneous_elasticity(n)
    m = p.mesh
    dofs = (3 * p.bc_nodes[:, None] + np.arange(3)).ravel().astype(np.int32)
    zval = np.zeros(dofs.size)
    S = fem.System(fem.ELASTIC, m.xyz, m.tets, m.mat)
    S.add_traction(p.faces, p.traction)
    S.assemble_elastic(p.E, p.nu)
    S.apply_dirichlet(dofs, zval, fem.ROW_AND_COLUMN)
    K = fem.System(fem.ELASTIC, m.xyz, m.tets, m.mat)
    K.assemble_elastic_textbook(p.E, p.nu)
    K.apply_dirichlet(dofs, zval, fem.ROW_AND_COLUMN)
    cc = meshgen.cube_cells(m, p.E, p.nu, 8)
    C = Cells(cc.cells)
    C.set_face_material("cells")
    rcb = C.build_bases(FP32_IR, 1e-8)
    T = TwoLevel(S, C, cc, dofs)
    if matrix_free:
        S.set_kuhn_grid(n)
        K.set_kuhn_grid(n)
        T.set_smoother(K, matrix_free=True)
        T.set_matrix_free(True)
    else:
        T.set_smoother(K, half_matrix=True)
    out_info = {}
    if smoother_reps:
        ms, nb = T.bench_smoother(reps=smoother_reps)
        out_info = {"smoother_ms": ms, "smoother_bytes": nb, "smoother_gbs": nb / (ms * 1e-3) / 1e9}
    rel, it, out, rc = T.solve(tol=1e-8, maxiter=maxiter, precision=FP64)
    print(json.dumps({"n": n, "dofs": S.n_rows, "matrix_free": matrix_free, "rc_bases": rcb, "rc": rc, "rel": rel,
                      "iterations": it, "ms_solve": S.stats()["ms_solve"], "coarse_setup_ms": T.ms_setup,
                      **out_info}))
    T.close()
    C.close()
    K.close()
    S.close()


def net_case(n):
    """The learned coarse space's prediction of n sphere cells (voxelisation, the 4 layers, the
    basis write) on each tensor-core path of layers 1-3, in path order 0 (mma.sync), 1, 2, 3
    (tcgen05): 2 warm-up predictions and 3 timed ones each (device ms from msfem_net_predict)."""
    import numpy as np

    from . import meshgen
    from .cells import Cells
    from .learned import CoarseNet
    net = CoarseNet(seed=0)
    C = Cells(meshgen.sphere_cells(n, seed=3))
    out = {"cells": n}
    for path in (0, 1, 2, 3):
        net.set_tensor_path(path)
        for _ in range(2):
            net.predict(C)
        ms = [net.predict(C) for _ in range(3)]
        out[f"path{path}"] = {"ms_predict_min": min(ms), "checksum": float(np.abs(C.bases()).sum())}
    print(json.dumps(out))
    net.close()
    C.close()


if __name__ == "__main__":
    main()
