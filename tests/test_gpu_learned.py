"""The learned coarse space on the GPU (multiscalefemsolver3d_b200/csrc/neural.cu through
learned.py) against its CPU restatement oracle/neural.py: voxelisation, forward pass, loss and
every layer's gradient on the same parameters and inputs; then what training buys: validation
loss against the trilinear coarse space, and two-level MINRES iterations with the predicted bases
against the trilinear ones.  The fallback re-solves exactly the cells it flags."""
import math

import numpy as np
import pytest

from multiscalefemsolver3d_b200 import fem, meshgen
from multiscalefemsolver3d_b200._lib import MsfemError
from multiscalefemsolver3d_b200.cells import FP32_IR, FP64, Cells
from multiscalefemsolver3d_b200.learned import CoarseNet, learned_bases, train_on_cells
from multiscalefemsolver3d_b200.twolevel import TwoLevel
from oracle import neural as on

pytestmark = pytest.mark.gpu

SCALE = 1.0 / math.log(100.0)


def _tet_values(cm):
    return SCALE * np.log(cm.E[cm.mat]).reshape(cm.n_cells, 3072)


@pytest.fixture(scope="module")
def trained(lib, cuda):
    net = CoarseNet(seed=0)
    info = train_on_cells(net, 2048, seed=1, epochs=12, batch=128, lr=1e-3)
    yield net, info
    net.close()


def test_voxelise_matches_oracle(lib, cuda):
    cm = meshgen.sphere_cells(5, seed=2)
    with_cells = Cells(cm)
    net = CoarseNet(seed=1)
    v = net.voxelise(with_cells)
    np.testing.assert_allclose(v, on.voxelise(_tet_values(cm)), rtol=0, atol=1e-6)
    # the exact share table: each voxel average of a constant is the constant
    assert np.all(v[cm.mat.reshape(5, -1).sum(axis=1) == 0] == 0)


def test_forward_and_gradients_match_oracle(lib, cuda):
    """Tolerances: BF16 storage points are reproduced by the oracle, so the two differ only by the
    FP32 accumulation order (and the rare BF16 rounding that order flips)."""
    p = on.init_params(3)
    net = CoarseNet()
    net.set_params(p)
    np.testing.assert_array_equal(net.params(), p)
    vox = on.voxelise(_tet_values(meshgen.sphere_cells(2, seed=4))).astype(np.float32)
    out = net.forward(vox)
    ref = on.forward(p, vox)
    for k in range(2):
        o = ref[k][1]
        assert np.linalg.norm(out[k] - o) <= 5e-3 * np.linalg.norm(o)
        assert np.abs(out[k] - o).max() <= 2e-2 * np.abs(o).max()
        assert np.all(out[k][:, 24:] == 0)
    rng = np.random.default_rng(0)
    tgt = rng.normal(0, 0.05, (2, 729, 24)).astype(np.float32)
    loss, g = net.loss_grad(vox, tgt)
    loss_ref, g_ref = on.loss_grad(p, vox, tgt)
    assert loss == pytest.approx(loss_ref, rel=1e-4)
    for lo, hi in [(0, on.L1), (on.layer_base(1), on.layer_base(2)), (on.layer_base(2), on.layer_base(3)),
                   (on.layer_base(3), on.PARAMS)]:
        assert np.linalg.norm(g[lo:hi] - g_ref[lo:hi]) <= 2e-3 * np.linalg.norm(g_ref[lo:hi])
    # deterministic: the same pass twice gives the same bits
    loss2, g2 = net.loss_grad(vox, tgt)
    assert loss2 == loss and np.array_equal(g, g2)


def test_training_beats_trilinear_on_new_cells(trained):
    net, info = trained
    assert info["cells"] == 2048 and np.all(np.isfinite(info["losses"]))
    cm = meshgen.sphere_cells(256, seed=99)
    C = Cells(cm)
    assert C.build_bases(FP32_IR, 1e-8) == 0
    target = (C.bases().reshape(-1, 729, 24) - on.q1()[None]).astype(np.float32)
    wild = np.abs(C.bases().reshape(-1, 729 * 24)).max(axis=1) > 3.0   # trilinear targets, as in training
    target[wild] = 0.0
    loss, _ = net.loss_grad(net.voxelise(C), target)
    assert loss < 0.85 * float((target.astype(np.float64) ** 2).mean())


def _elastic_case(n=32):
    p = meshgen.cube_elastic(n=n, jitter=0.0, n_spheres=31, contrast=100.0, rmin=0.06, rmax=0.14, sphere_seed=11)
    m = p.mesh
    dofs = (3 * p.bc_nodes[:, None] + np.arange(3)).ravel().astype(np.int32)
    z = np.zeros(dofs.size)
    S = fem.System(fem.ELASTIC, m.xyz, m.tets, m.mat)
    S.add_traction(p.faces, p.traction)
    S.assemble_elastic(p.E, p.nu)
    S.apply_dirichlet(dofs, z, fem.ROW_AND_COLUMN)
    K = fem.System(fem.ELASTIC, m.xyz, m.tets, m.mat)
    K.assemble_elastic_textbook(p.E, p.nu)
    K.apply_dirichlet(dofs, z, fem.ROW_AND_COLUMN)
    return S, K, meshgen.cube_cells(m, p.E, p.nu, 8), dofs


def _iterations(S, K, cc, dofs, C):
    T = TwoLevel(S, C, cc, dofs)
    T.set_smoother(K, degree=3, ratio=30.0, half_matrix=True)
    S.set_x(np.zeros(S.n_rows))
    rel, it, _, rc = T.solve(tol=1e-8, maxiter=100000, precision=FP64)
    T.close()
    assert rc == 0 and rel <= 1e-8
    return it


def test_learned_coarse_space_cuts_iterations(trained):
    """The gain over the method without the network: the same two-level solve with the trilinear
    coarse space (an all-zero network predicts exactly Q1) needs more iterations."""
    net, _ = trained
    S, K, cc, dofs = _elastic_case()
    zero = CoarseNet()
    zero.set_params(np.zeros(zero.n_params, np.float32))
    Cq = Cells(cc.cells)
    zero.predict(Cq)
    q = Cq.bases().reshape(-1, 729, 24)
    np.testing.assert_allclose(q, np.broadcast_to(on.q1(), q.shape), rtol=0, atol=1e-7)
    it_q1 = _iterations(S, K, cc, dofs, Cq)
    Cl = Cells(cc.cells)
    info = learned_bases(net, Cl, cc.cells)
    it_learned = _iterations(S, K, cc, dofs, Cl)
    assert info["fallback_cells"] <= cc.cells.n_cells // 4
    assert it_learned < 0.8 * it_q1, (it_learned, it_q1)


def test_fallback_replaces_flagged_cells_with_exact_bases(lib, cuda):
    cm = meshgen.sphere_cells(12, seed=5)
    Ce = Cells(cm)
    assert Ce.build_bases(FP64, 1e-12) == 0
    exact = Ce.bases()
    assert np.all(Ce.basis_residual() < 1e-9)
    net = CoarseNet(seed=3)                       # untrained: every prediction is poor
    C = Cells(cm)
    info = learned_bases(net, C, cm, threshold=0.0, precision=FP64, tol=1e-12)
    assert info["fallback_cells"] == 12
    np.testing.assert_allclose(C.bases(), exact, rtol=0, atol=1e-9)
    C2 = Cells(cm)
    info = learned_bases(net, C2, cm, threshold=np.inf)
    assert info["fallback_cells"] == 0 and np.all(info["residual"] > 1e-3)


def test_rejects_cells_that_are_not_kuhn_cubes_of_8(lib, cuda):
    cm = meshgen.msfem_cells(n_coarse=2, m_choices=(6,), seed=1)
    C = Cells(cm)
    net = CoarseNet()
    with pytest.raises(MsfemError, match="8 x 8 x 8 Kuhn cube"):
        net.voxelise(C)
    C.close()
    net.close()


def test_tcgen05_path_matches_mma_sync(lib, cuda):
    """Layers 1-3 on tcgen05 (TMEM accumulators, shared-memory descriptors; voxel-tile, transposed
    and warp-specialised persistent forms) compute the same function as the warp-level mma.sync
    kernels: forward outputs, loss and every gradient."""
    p = on.init_params(5)
    net = CoarseNet()
    net.set_params(p)
    vox = on.voxelise(_tet_values(meshgen.sphere_cells(3, seed=8))).astype(np.float32)
    tgt = np.random.default_rng(2).normal(0, 0.05, (3, 729, 24)).astype(np.float32)
    net.set_tensor_path(0)
    o_ref = net.forward(vox)
    l_ref, g_ref = net.loss_grad(vox, tgt)
    ref = on.forward(p, vox)
    for path in (1, 2, 3):
        net.set_tensor_path(path)
        o_tc = net.forward(vox)
        l_tc, g_tc = net.loss_grad(vox, tgt)
        assert np.linalg.norm(o_tc - o_ref) <= 1e-5 * np.linalg.norm(o_ref), path
        assert l_tc == pytest.approx(l_ref, rel=1e-5)
        assert np.linalg.norm(g_tc - g_ref) <= 1e-4 * np.linalg.norm(g_ref), path
        for k in range(3):
            assert np.linalg.norm(o_tc[k] - ref[k][1]) <= 5e-3 * np.linalg.norm(ref[k][1])


def test_persistent_tcgen05_path_over_many_cells(lib, cuda):
    """The warp-specialised tcgen05 kernel walks several cells per CTA (a ring of plane slots and
    two TMEM accumulators carried across cells): 400 cells (more than one per SM) give the
    mma.sync path's forward output."""
    net = CoarseNet()
    net.set_params(on.init_params(7))
    vox = np.random.default_rng(3).normal(0.0, 1.0, (400, 4096)).astype(np.float32)
    net.set_tensor_path(0)
    o_ref = net.forward(vox)
    net.set_tensor_path(3)
    o_ws = net.forward(vox)
    assert np.linalg.norm(o_ws - o_ref) <= 1e-5 * np.linalg.norm(o_ref)
    for k in (0, 147, 148, 399):
        assert np.linalg.norm(o_ws[k] - o_ref[k]) <= 1e-5 * np.linalg.norm(o_ref[k]), k

