"""Test infrastructure only: CPU restatement (numpy, float64) of the learned coarse space's
network -- voxelisation, forward pass, loss, and the hand-derived backward pass -- used to check
the GPU kernels of multiscalefemsolver3d_b200/csrc/neural.cu.  The reference has no learned
component; the network is this project's own, so parity here means "the GPU computes this
function and its exact gradient".

`bf16=True` rounds at the points where the GPU stores BF16 (the weights of layers 1-3, the
activations after each ReLU, the loss gradient entering layer 3, and each masked data gradient),
so that GPU and oracle differ only by FP32 accumulation order; `bf16=False` is the exact float64
function, which tests/test_neural_oracle.py checks against finite differences.

Parameter layout (float32 vector of PARAMS entries):
  W0 [27][32][4], b0 [32], then for l = 1..3: W_l [27][32 co][32 ci], b_l [32]
  (layer 3 uses output channels 0..23; rows 24..31 are zero).
Taps: t = 9 dz + 3 dy + dx, offset (dz-1, dy-1, dx-1) in (z, y, x); voxel v = (z*16 + y)*16 + x.
"""
from __future__ import annotations

import numpy as np

V, VOX, N, NODES, CH, OUT, TAPS, CIN0 = 16, 4096, 9, 729, 32, 24, 27, 4
W0 = 0
B0 = TAPS * CH * CIN0
L1 = B0 + CH
LAYERW = TAPS * CH * CH
LAYER = LAYERW + CH
PARAMS = L1 + 3 * LAYER

KUHN_ORDER = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]


def layer_base(l):
    return L1 + (l - 1) * LAYER


def bf16(a):
    """Round to bfloat16 (through float32, round to nearest even), returned as float64."""
    f = np.asarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def kuhn_share(oct_, t):
    """Share of octant oct_ of a hexahedron inside Kuhn tetrahedron t (see csrc/neural.cu)."""
    h = [oct_ & 1, (oct_ >> 1) & 1, (oct_ >> 2) & 1]
    ok = [h[o[0]] >= h[o[1]] >= h[o[2]] for o in KUHN_ORDER]
    return (1.0 / sum(ok)) if ok[t] else 0.0


def voxelise(tet_values):
    """tet_values [n, 3072] (s ln(E/E_ref) of each tetrahedron in Kuhn-cube order) -> [n, 4096]."""
    tv = np.asarray(tet_values, dtype=np.float64)
    share = np.array([[kuhn_share(o, t) for t in range(6)] for o in range(8)])
    z, y, x = np.meshgrid(np.arange(V), np.arange(V), np.arange(V), indexing="ij")
    z, y, x = z.ravel(), y.ravel(), x.ravel()
    hexi = (x >> 1) + 8 * ((y >> 1) + 8 * (z >> 1))
    oct_ = (x & 1) | ((y & 1) << 1) | ((z & 1) << 2)
    tets = 6 * hexi[:, None] + np.arange(6)[None, :]          # [4096, 6]
    return np.einsum("vt,nvt->nv", share[oct_], tv[:, tets])


def _coords():
    z, y, x = np.meshgrid(np.arange(V), np.arange(V), np.arange(V), indexing="ij")
    c = lambda i: (2.0 * i + 1.0) / V - 1.0  # noqa: E731
    return np.stack([c(x.ravel()), c(y.ravel()), c(z.ravel())], axis=1)


def _patches(a):
    """a [4096, C] -> [4096, 27, C] (zero outside the cell)."""
    C = a.shape[1]
    g = np.zeros((V + 2, V + 2, V + 2, C))
    g[1:-1, 1:-1, 1:-1] = a.reshape(V, V, V, C)
    out = np.empty((VOX, TAPS, C))
    for t in range(TAPS):
        dz, dy, dx = t // 9, (t // 3) % 3, t % 3
        out[:, t] = g[dz:dz + V, dy:dy + V, dx:dx + V].reshape(VOX, C)
    return out


def _unpack(p, rounded):
    p = np.asarray(p, dtype=np.float64)
    w0 = p[W0:W0 + B0].reshape(TAPS, CH, CIN0)
    b0 = p[B0:B0 + CH]
    Ws, bs = [], []
    for l in (1, 2, 3):
        w = p[layer_base(l):layer_base(l) + LAYERW].reshape(TAPS, CH, CH)
        Ws.append(bf16(w) if rounded else w)
        bs.append(p[layer_base(l) + LAYERW:layer_base(l) + LAYER])
    return w0, b0, Ws, bs


def _node_maps():
    i = np.arange(V)
    node_of = (i + 1) >> 1                                     # per axis
    z, y, x = np.meshgrid(i, i, i, indexing="ij")
    node = (node_of[x] + N * (node_of[y] + N * node_of[z])).ravel()
    cnt1 = np.where((np.arange(N) == 0) | (np.arange(N) == N - 1), 1, 2)
    k, j, ii = np.meshgrid(np.arange(N), np.arange(N), np.arange(N), indexing="ij")
    cnt = (cnt1[ii] * cnt1[j] * cnt1[k]).ravel()
    vert = (np.isin(ii, [0, N - 1]) & np.isin(j, [0, N - 1]) & np.isin(k, [0, N - 1])).ravel()
    return node, cnt, vert


def q1():
    """[729, 24]: the trilinear functions, channel 3 v + a."""
    k, j, i = np.meshgrid(np.arange(N), np.arange(N), np.arange(N), indexing="ij")
    t = [i.ravel() / 8.0, j.ravel() / 8.0, k.ravel() / 8.0]
    out = np.empty((NODES, OUT))
    for v in range(8):
        f = np.ones(NODES)
        for d in range(3):
            f = f * (t[d] if (v >> d) & 1 else 1.0 - t[d])
        out[:, 3 * v:3 * v + 3] = f[:, None]
    return out


def forward(p, vox, bf16_points=True):
    """Per cell: (activations list, output [4096, 32]).  vox [n, 4096]."""
    w0, b0, Ws, bs = _unpack(p, bf16_points)
    R = bf16 if bf16_points else (lambda a: a)
    coords = _coords()
    res = []
    for x in np.asarray(vox, dtype=np.float64):
        inp = np.concatenate([x[:, None], coords], axis=1)
        P0 = _patches(inp)
        a0 = R(np.maximum(np.einsum("vtc,toc->vo", P0, w0) + b0, 0.0))
        acts = [inp, a0]
        a = a0
        for l in range(3):
            P = _patches(a).reshape(VOX, TAPS * CH)
            z = P @ Ws[l].transpose(0, 2, 1).reshape(TAPS * CH, CH) + bs[l]
            if l < 2:
                a = R(np.maximum(z, 0.0))
                acts.append(a)
            else:
                a = z
        res.append((acts, a))
    return res


def node_corr(o):
    """o [4096, 32] -> corr [729, 24] (zero at the 8 cell vertices)."""
    node, cnt, vert = _node_maps()
    s = np.zeros((NODES, OUT))
    np.add.at(s, node, o[:, :OUT])
    s /= cnt[:, None]
    s[vert] = 0.0
    return s


def loss_grad(p, vox, target, bf16_points=True):
    """(loss, grad [PARAMS]) of the mean square (corr - target) over cells, nodes and channels."""
    w0, b0, Ws, bs = _unpack(p, bf16_points)
    R = bf16 if bf16_points else (lambda a: a)
    node, cnt, vert = _node_maps()
    target = np.asarray(target, dtype=np.float64).reshape(-1, NODES, OUT)
    n = target.shape[0]
    inv = 1.0 / (n * NODES * OUT)
    g = np.zeros(PARAMS)
    loss = 0.0
    for (acts, o), y in zip(forward(p, vox, bf16_points), target):
        d = node_corr(o) - y
        loss += (d * d).sum()
        gn = 2.0 * d * inv / cnt[:, None]
        gn[vert] = 0.0
        dz = np.zeros((VOX, CH))
        dz[:, :OUT] = gn[node]
        dz = R(dz)
        for l in (3, 2, 1):
            a_in = acts[l]                                  # input of layer l (a0, a1, a2)
            P = _patches(a_in)                              # [4096, 27, 32]
            g[layer_base(l):layer_base(l) + LAYERW] += np.einsum("vo,vti->toi", dz, P).ravel()
            g[layer_base(l) + LAYERW:layer_base(l) + LAYER] += dz.sum(axis=0)
            W = Ws[l - 1]                                   # [27][co][ci]
            Q = _patches(dz)                                # dz at v + offset(t')
            da = np.einsum("vto,toi->vi", Q, W[::-1])       # W[26 - t']
            dz = R(da * (a_in > 0))
        P0 = _patches(acts[0])
        g[W0:W0 + B0] += np.einsum("vo,vtc->toc", dz, P0).ravel()
        g[B0:B0 + CH] += dz.sum(axis=0)
    return loss * inv, g


def init_params(seed=0):
    """Random parameters in the GPU's layout (not the GPU's generator; for tests)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(PARAMS)
    p[W0:B0] = rng.uniform(-1, 1, B0) * np.sqrt(6.0 / (TAPS * CIN0))
    p[B0:B0 + CH] = rng.uniform(-0.1, 0.1, CH)
    for l in (1, 2, 3):
        w = rng.uniform(-1, 1, (TAPS, CH, CH)) * np.sqrt(6.0 / (TAPS * CH))
        b = rng.uniform(-0.1, 0.1, CH)
        if l == 3:
            w[:, OUT:, :] = 0.0
            b[OUT:] = 0.0
        p[layer_base(l):layer_base(l) + LAYERW] = w.ravel()
        p[layer_base(l) + LAYERW:layer_base(l) + LAYER] = b
    return p.astype(np.float32)
