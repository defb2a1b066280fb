"""Learned MsFEM coarse space (include/msfem_b200.h, msfem_net_*): a 3D convolutional operator
that predicts each macro cell's Order1 bases from its voxelised Young's-modulus field, trained on
the bases that the batched cell solver computes, and the coarse-space builder that uses it with
the exact cell solve as the per-cell fallback.  Every kernel runs in libmsfem_b200.so.

The reference's bases always come from its cell problems (MsFEM_Grid.h,
Grid_forMech_Poly_Order1::CreateFunctionalSpaces); the predicted ones only enter the two-level
preconditioner (twolevel.TwoLevel), so a poor prediction costs Krylov iterations, not accuracy.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np

from . import meshgen
from ._lib import FP32_IR, check, load
from .cells import Cells

__all__ = ["CoarseNet", "learned_bases", "PARAMS"]


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def __getattr__(name):
    if name == "PARAMS":
        return load().msfem_net_param_count()
    raise AttributeError(name)


class CoarseNet:
    """The network and its training set on the GPU.

    E_ref, in_scale: the input is in_scale * ln(E / E_ref) averaged over each voxel (defaults:
    E_ref = 1, in_scale = 1 / ln 100, so a 1:100 inclusion reads 1)."""

    def __init__(self, seed: int = 0, E_ref: float = 1.0, in_scale: float = 1.0 / math.log(100.0)):
        L = load()
        h = C.c_void_p()
        check(L.msfem_net_create(seed, E_ref, in_scale, C.byref(h)), "net_create")
        self.h = h
        self.n_params = L.msfem_net_param_count()
        self.n_train = 0

    def set_tensor_path(self, path: int):
        """Layers 1-3: 0 = warp-level mma.sync, 1 = tcgen05 with M = 64 voxel tiles, 2 = tcgen05
        transposed product (N = 256 voxels per instruction), 3 = tcgen05 with M = 64 voxel tiles,
        warp-specialised (load / MMA / epilogue warps) and persistent over cells."""
        check(load().msfem_net_set_tensor_path(self.h, int(path)), "net_set_tensor_path")

    def params(self) -> np.ndarray:
        p = np.empty(self.n_params, np.float32)
        check(load().msfem_net_get_params(self.h, _p(p)), "net_get_params")
        return p

    def set_params(self, p):
        p = _c(p, np.float32)
        if p.size != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters")
        check(load().msfem_net_set_params(self.h, _p(p)), "net_set_params")

    def voxelise(self, cells: Cells) -> np.ndarray:
        out = np.empty((cells.n_cells, 4096), np.float32)
        check(load().msfem_net_voxelise(self.h, cells.h, _p(out)), "net_voxelise")
        return out

    def add_cells(self, cells: Cells) -> int:
        """Adds every cell of `cells` (bases built) to the training set; returns its size."""
        n = C.c_int()
        check(load().msfem_net_add_cells(self.h, cells.h, C.byref(n)), "net_add_cells")
        self.n_train = n.value
        return n.value

    def train(self, steps: int, batch: int = 128, lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        losses = np.empty(steps, np.float32)
        check(load().msfem_net_train(self.h, steps, batch, lr, seed, _p(losses)), "net_train")
        return losses

    def loss_grad(self, vox, target):
        vox = _c(vox, np.float32)
        target = _c(target, np.float32)
        n = vox.shape[0]
        loss = np.zeros(1, np.float32)
        g = np.empty(self.n_params, np.float32)
        check(load().msfem_net_loss_grad(self.h, n, _p(vox), _p(target), _p(loss), _p(g)), "net_loss_grad")
        return float(loss[0]), g

    def forward(self, vox) -> np.ndarray:
        vox = _c(vox, np.float32)
        out = np.empty((vox.shape[0], 4096, 32), np.float32)
        check(load().msfem_net_forward(self.h, vox.shape[0], _p(vox), _p(out)), "net_forward")
        return out

    def predict(self, cells: Cells) -> float:
        """Writes the predicted bases of every cell into `cells`; returns the device ms."""
        ms = np.zeros(1, np.float32)
        check(load().msfem_net_predict(self.h, cells.h, _p(ms)), "net_predict")
        return float(ms[0])

    def close(self):
        if getattr(self, "h", None):
            load().msfem_net_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def train_on_cells(net: CoarseNet, n_cells: int, seed: int = 0, chunk: int = 4096, epochs: int = 20, batch: int = 128,
                   lr: float = 2e-3, face_material: str = "zero", **cell_kw) -> dict:
    """Generates n_cells training cells (meshgen.sphere_cells), solves their exact bases with the
    batched cell solver (face and edge problems on `face_material`, Cells.set_face_material), adds
    them to the training set and trains `epochs` passes with a cosine learning-rate decay.  Returns
    timings and the loss curve."""
    t0 = time.perf_counter()
    ms_solve = 0.0
    for k, c0 in enumerate(range(0, n_cells, chunk)):
        cm = meshgen.sphere_cells(min(chunk, n_cells - c0), seed=seed * 1000 + k, **cell_kw)
        cells = Cells(cm)
        cells.set_face_material(face_material)
        rc = cells.build_bases(FP32_IR, 1e-8)
        if rc != 0:
            raise RuntimeError(f"training cells: bases rc={rc}")
        ms_solve += sum(cells.report()["ms"].values())
        net.add_cells(cells)
        cells.close()
    t_data = time.perf_counter() - t0
    steps_per_epoch = max(1, net.n_train // batch)
    total = epochs * steps_per_epoch
    losses = []
    t1 = time.perf_counter()
    rounds = 10
    for r in range(rounds):
        lr_r = lr * 0.5 * (1.0 + math.cos(math.pi * r / rounds))
        n = total // rounds + (1 if r < total % rounds else 0)
        if n:
            losses.append(net.train(n, batch=batch, lr=lr_r, seed=seed * 7919 + r))
    t_train = time.perf_counter() - t1
    return {"cells": net.n_train, "ms_cell_solves": ms_solve, "s_data": t_data, "s_train": t_train,
            "steps": total, "losses": np.concatenate(losses) if losses else np.zeros(0, np.float32)}


def learned_bases(net: CoarseNet, cells: Cells, cell_meshes, threshold: float = 1.0, precision=FP32_IR,
                  tol: float = 1e-8, face_material: str = "zero") -> dict:
    """Predicted bases for every cell of `cells`; each cell whose predicted bases leave a volume
    residual above `threshold` (Cells.basis_residual) is re-solved exactly (the batched cell
    solver on those cells only) and its exact bases replace the prediction.  The default 1.0 is
    the residual of the trivial interior extension (psi_I = 0): only predictions worse than that
    fall back.  A lower threshold is not better by itself -- on the sphere workloads the exact
    MsFEM bases make a weaker coarse space for the textbook-operator cycle than the predicted
    ones, so replacing moderately wrong predictions raised the iteration count.  face_material: the
    convention of the exact fallback solves (as the network's training targets were made)."""
    t0 = time.perf_counter()
    ms_pred = net.predict(cells)
    rel = cells.basis_residual()
    bad = np.nonzero(~(rel <= threshold))[0].astype(np.int32)
    ms_fallback = 0.0
    if bad.size:
        sub = Cells(meshgen.subset_cells(cell_meshes, bad))
        sub.set_face_material(face_material)
        rc = sub.build_bases(precision, tol)
        if rc != 0:
            raise RuntimeError(f"fallback cells: bases rc={rc}")
        ms_fallback = sum(sub.report()["ms"].values())
        cells.copy_bases_from(sub, bad)
        sub.close()
    return {"ms_predict": ms_pred, "ms_fallback": ms_fallback, "fallback_cells": int(bad.size),
            "residual": rel, "s_total": time.perf_counter() - t0}
