"""Matrix-free Newton-Raphson with load stepping over the engine.

The reference's canonical driver (HyperFEMKernels ``test/solvers/test_pmultigrid.jl:86-115``; in
production HyperFEM's ``NewtonRaphson``, ``benchmark/solvers/krylov.jl:194-202``): per Newton
iteration ``residual!``, ``jacobian!(mf, op, x)`` (prepare), ``numerical_setup!`` (the p-multigrid
levels follow the state) and ``solve!`` with ``MatrixFreeSolver``; the Dirichlet values of the
loaded face scale with the load factor. The state, residual and increments stay on the GPU when
torch is available (device pointers through the C ABI).
"""
from __future__ import annotations

import dataclasses
import time

import numpy as np

from . import solvers as S
from .operator import KernelOperator


@dataclasses.dataclass
class NewtonStats:
    load_steps: int = 0
    newton_iters: int = 0
    krylov_iters: list = dataclasses.field(default_factory=list)
    residual_norms: list = dataclasses.field(default_factory=list)
    converged: bool = True
    seconds: float = 0.0
    pmg: dict = None  # p-multigrid counters and times (PMultigridState.stats)


def newton_solve(op: KernelOperator, solver: S.MatrixFreeSolver, g_full: np.ndarray, loads, x0=None, *,
                 rtol_newton=1e-8, atol_newton=1e-12, max_newton=20, device=True, lift=None):
    """Solve R(x; load * g_full) = 0 for each load factor in ``loads`` (continuation from the previous one).

    ``g_full`` are the Dirichlet values at load factor 1. Returns (x, NewtonStats). Newton stops when
    ||R|| <= max(rtol_newton * ||R_0||, atol_newton), R_0 the residual at the first iterate of the step.
    ``lift`` (free dofs, at load factor 1): a field that carries the Dirichlet data into the interior;
    each load step then starts from x + (load increment) * lift (no strain jump at the loaded
    boundary in the step's first tangent). None keeps x, as the reference's loop does.
    """
    import torch

    U = op.U
    n = U.nfree
    dev = torch.device("cuda") if device else None
    x = torch.zeros(n, dtype=torch.float64, device=dev) if x0 is None else torch.as_tensor(x0, device=dev).clone()
    b = torch.zeros(n, dtype=torch.float64, device=dev)
    dx = torch.zeros(n, dtype=torch.float64, device=dev)
    mf = op.allocate_jacobian(x)
    ns = None
    st = NewtonStats()
    lift_d = None if lift is None else torch.as_tensor(np.ascontiguousarray(lift, dtype=float), device=dev)
    prev = 0.0
    t0 = time.perf_counter()
    for lam in loads:
        U.dirichlet_values = np.ascontiguousarray(lam * g_full)
        dv = torch.as_tensor(U.dirichlet_values, device=dev)
        if lift_d is not None:
            x += (lam - prev) * lift_d
        prev = lam
        st.load_steps += 1
        r0 = None
        for it in range(max_newton):
            op.residual(b, x, dv)
            rn = float(torch.linalg.norm(b))
            st.residual_norms.append(rn)
            if r0 is None:
                r0 = rn
            if rn <= max(rtol_newton * r0, atol_newton):
                break
            mf.prepare(x, dv)
            if ns is None:
                ns = S.numerical_setup(S.symbolic_setup(solver, mf), mf)
            else:
                S.numerical_setup_update(ns, mf)
            dx.zero_()
            b.neg_()
            S.solve(dx, ns, b)
            st.krylov_iters.append(S.linear_iterations(ns))
            if not S.linear_converged(ns):
                st.converged = False
                break
            x += dx
            st.newton_iters += 1
        else:
            st.converged = False
        if not st.converged:
            break
    torch.cuda.synchronize()
    st.seconds = time.perf_counter() - t0
    if ns is not None and ns.prec is not None and hasattr(ns.prec, "stats"):
        st.pmg = ns.prec.stats()
    return x, st
