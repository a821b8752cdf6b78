import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "hyperfemkernels.jl_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libhfk.so")


def has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA GPU in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def svk_space(n=(3, 2, 2), order=2, perturb=0.0, seed=3, disp=0.05, faces=("x0", "x1")):
    """Cube of Q_order hexahedra, x0 clamped, x1 displaced `disp` in x (the SVK benchmark setting)."""
    from hfk.fespace import CartesianMesh, VectorLagrangeSpace

    m = CartesianMesh(n, perturb=perturb, seed=seed)
    g = [lambda x: 0 * x, lambda x: np.tile([disp, 0.0, 0.0], (len(x), 1))]
    if faces != ("x0", "x1"):
        g = lambda x: np.stack([0.01 * x[:, 0], -0.02 * x[:, 1] * x[:, 2], 0.005 + 0 * x[:, 0]], axis=1)
    return VectorLagrangeSpace(m, order, faces, g=g)


def svk_state(V, seed=0, amp=1e-3, disp=0.05):
    """u = disp*x e_x + seeded uniform perturbation (+-amp) on free dofs."""
    rng = np.random.default_rng(seed)
    free, _ = V.interpolate(lambda x: np.stack([disp * x[:, 0], 0 * x[:, 0], 0 * x[:, 0]], axis=1))
    return free + rng.uniform(-amp, amp, V.nfree)


def reldiff(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)
