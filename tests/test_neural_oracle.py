"""The learned coarse space's CPU restatement (oracle/neural.py): its hand-derived gradient
against central finite differences of its own float64 loss, layer by layer, and the exactness
of the voxelisation (Kuhn-tetrahedron shares of each voxel)."""
import numpy as np
import pytest

from oracle import neural as on


def _case(seed=0, n=1):
    rng = np.random.default_rng(seed)
    vox = rng.uniform(0.0, 1.0, (n, on.VOX))
    target = rng.normal(0.0, 0.05, (n, on.NODES, on.OUT))
    return on.init_params(seed).astype(np.float64), vox, target


@pytest.mark.parametrize("block", ["L0", "L1", "L2", "L3"])
def test_oracle_gradient_matches_finite_differences(block):
    p, vox, target = _case(1)
    lo, hi = {"L0": (0, on.L1), "L1": (on.layer_base(1), on.layer_base(2)),
              "L2": (on.layer_base(2), on.layer_base(3)), "L3": (on.layer_base(3), on.PARAMS)}[block]
    rng = np.random.default_rng(7)
    d = np.zeros(on.PARAMS)
    d[lo:hi] = rng.normal(size=hi - lo)
    if block == "L3":   # padded output rows stay zero
        w = d[lo:lo + on.LAYERW].reshape(on.TAPS, on.CH, on.CH)
        w[:, on.OUT:, :] = 0.0
        d[lo + on.LAYERW + on.OUT:hi] = 0.0
    d /= np.linalg.norm(d)
    _, g = on.loss_grad(p, vox, target, bf16_points=False)
    eps = 1e-6   # small enough that no ReLU changes sign between p - eps d and p + eps d
    lp, _ = on.loss_grad(p + eps * d, vox, target, bf16_points=False)
    lm, _ = on.loss_grad(p - eps * d, vox, target, bf16_points=False)
    fd = (lp - lm) / (2 * eps)
    assert abs(g @ d - fd) <= 1e-6 * abs(fd) + 1e-12


def test_voxelise_shares_are_exact():
    share = np.array([[on.kuhn_share(o, t) for t in range(6)] for o in range(8)])
    np.testing.assert_allclose(share.sum(axis=1), 1.0)          # each octant is covered once
    np.testing.assert_allclose(share.sum(axis=0), 8.0 / 6.0)    # each tet is 1/6 of the hexahedron
    rng = np.random.default_rng(3)
    tv = rng.normal(size=(2, 3072))
    v = on.voxelise(tv)
    np.testing.assert_allclose(v.mean(axis=1), tv.mean(axis=1), rtol=0, atol=1e-14)
    np.testing.assert_allclose(on.voxelise(np.full((1, 3072), 0.7)), 0.7, rtol=0, atol=1e-15)


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -2.5, 1e-30, 3.0e38])
    r = on.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2.0 ** -6 and r[3] == -2.5
    assert abs(r[4] - 1e-30) <= 1e-30 * 2 ** -8
    q = on.q1()
    np.testing.assert_allclose(q.reshape(729, 8, 3).sum(axis=1), 1.0)
