"""Learned correction for the p-multigrid V-cycle (no counterpart in the reference).

A per-node MLP (16 -> 64 -> 64 -> 3, BF16 weights, FP32 accumulation; ``libhfk`` kernels for the
forward pass, the gradient and Adam) predicts the error left by the plain V-cycle from local
features of the residual. Inside the cycle the prediction delta is added with the per-problem step
that minimises the energy error along it (zero when delta is not a descent direction), so the plain
cycle remains the fallback (``hfk_pmg_set_mlp``). Training pairs come from
the plain cycle on seeded states (``hfk_pmg_mlp_sample``: target = the exact remaining error).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import call, ptr


def num_params() -> int:
    return int(_lib.lib().hfk_mlp_num_params())


class MLP:
    """The network handle (``hfk_mlp``)."""

    NIN, WIDTH, NOUT = 16, 64, 3

    def __init__(self, seed: int = 0):
        h = ctypes.c_void_p()
        call("hfk_mlp_create", ctypes.byref(h), ctypes.c_uint64(seed))
        self.h = h

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            try:
                _lib.lib().hfk_mlp_destroy(h)
            except Exception:
                pass
            self.h = None

    def weights(self) -> np.ndarray:
        w = np.zeros(num_params(), dtype=np.float32)
        call("hfk_mlp_get_weights", self.h, ptr(w, np.float32))
        return w

    def set_weights(self, w: np.ndarray):
        w = np.ascontiguousarray(w, dtype=np.float32)
        call("hfk_mlp_set_weights", self.h, ptr(w, np.float32))

    def forward(self, feats, out):
        """out (n x 3) = MLP(feats (n x 16)); CUDA float32 tensors."""
        call("hfk_mlp_forward", self.h, ptr(feats, np.float32), feats.shape[0], ptr(out, np.float32))
        return out

    def grad(self, feats, targets):
        g = np.zeros(num_params(), dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        call("hfk_mlp_grad", self.h, ptr(feats, np.float32), ptr(targets, np.float32), feats.shape[0],
             ptr(g, np.float32), ptr(loss, np.float32))
        return g, float(loss[0])

    def train(self, feats, targets, steps: int, batch: int = 4096, lr: float = 1e-3) -> float:
        loss = np.zeros(1, dtype=np.float32)
        call("hfk_mlp_train", self.h, ptr(feats, np.float32), ptr(targets, np.float32), feats.shape[0], steps, batch,
             ctypes.c_float(lr), ptr(loss, np.float32))
        return float(loss[0])


def collect_samples(pmg_state, mf, rhs, cycles: int = 3, rtol: float = 1e-10):
    """Training samples from the plain cycle: residuals of the stationary iteration
    r_{j+1} = r_j - A V(r_j) from ``rhs`` (a CUDA float64 tensor), ``cycles`` sets of
    (features, targets) per call. Returns CUDA float32 tensors (n x 16), (n x 3)."""
    import torch

    n = rhs.numel()
    feats, targets = [], []
    r = rhs.clone()
    y = torch.zeros_like(r)
    Ay = torch.zeros_like(r)
    nb = pmg_state.problems[0].space.nnodes  # an upper bound of the nodal blocks
    for _ in range(cycles):
        f = torch.zeros(nb, 16, dtype=torch.float32, device=r.device)
        t = torch.zeros(nb, 3, dtype=torch.float32, device=r.device)
        ns = ctypes.c_int()
        call("hfk_pmg_mlp_sample", pmg_state.h, ptr(r), ptr(f, np.float32), ptr(t, np.float32), ctypes.byref(ns), rtol)
        feats.append(f[: ns.value].clone())
        targets.append(t[: ns.value].clone())
        pmg_state.ldiv(y, r)
        mf.mul(Ay, y)
        r = r - Ay
    return torch.cat(feats), torch.cat(targets)


def attach(pmg_state, net: MLP | None):
    call("hfk_pmg_set_mlp", pmg_state.h, net.h if net is not None else None)
    pmg_state.mlp = net


def stats(pmg_state):
    tried, acc = ctypes.c_int64(), ctypes.c_int64()
    call("hfk_pmg_mlp_stats", pmg_state.h, ctypes.byref(tried), ctypes.byref(acc))
    return {"tried": tried.value, "accepted": acc.value}
