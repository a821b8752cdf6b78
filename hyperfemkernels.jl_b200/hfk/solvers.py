"""Solver layer: ``BlockJacobi``, ``Chebyshev``, ``Prolongation``, ``PMultigrid``, ``MatrixFreeSolver``.

Mirrors the reference's solver API (HyperFEMKernels ``src/preconditioners.jl``, ``src/smoothers.jl``,
``src/transfers.jl``, ``src/pmultigrid.jl``, ``src/solvers.jl``) over the engine: the smoothers,
V-cycle and Krylov iterations run on the GPU (``hfk_pmg_*``, ``hfk_solve_cg``). The Krylov method is
an FP64 (flexible) CG with the true-residual stopping test ``||b - J x|| <= atol + rtol ||b||``.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math

import numpy as np

from . import _lib
from ._lib import call, ptr
from .fespace import VectorLagrangeSpace, transfer_matrices
from .operator import KernelOperator, MatrixFreeJacobian, Problem


@dataclasses.dataclass(frozen=True)
class Chebyshev:
    """``Chebyshev(; degree = 2, range = 20.0, inflate = 1.1, eig_iters = 10)`` (src/smoothers.jl:21-33).

    ``eig_inner`` (an option of this engine): "euclidean" is the reference's Arnoldi estimate;
    "preconditioner" runs it in the P^-1 inner product, where J P^-1 is self-adjoint and the Ritz
    values stay inside the spectrum (a Lanczos estimate).
    """

    degree: int = 2
    range: float = 20.0
    inflate: float = 1.1
    eig_iters: int = 10
    eig_inner: str = "euclidean"

    def __post_init__(self):
        if self.degree < 1:
            raise ValueError("HyperFEMKernels: Chebyshev: degree must be ≥ 1")
        if not self.range > 1:
            raise ValueError("HyperFEMKernels: Chebyshev: range must be > 1")
        if self.inflate < 1:
            raise ValueError("HyperFEMKernels: Chebyshev: inflate must be ≥ 1")
        if self.eig_iters < 2:
            raise ValueError("HyperFEMKernels: Chebyshev: eig_iters must be ≥ 2")
        if self.eig_inner not in ("euclidean", "preconditioner"):
            raise ValueError("HyperFEMKernels: Chebyshev: eig_inner must be 'euclidean' or 'preconditioner'")


def chebyshev_damping(c: Chebyshev) -> float:
    """Damping of the smoother on its interval, 1/T_k(theta/delta) (src/smoothers.jl:35-40)."""
    b = 1.0
    a = b / c.range
    th, de = (b + a) / 2, (b - a) / 2
    return 1.0 / math.cosh(c.degree * math.acosh(th / de))


def chebyshev_start(n: int) -> np.ndarray:
    """Fixed start vector of the eigenvalue estimate (src/smoothers.jl:68-71)."""
    i = np.arange(1, n + 1, dtype=float)
    v = np.sin(1.0 + 0.7 * i) + 0.3 * np.cos(2.3 * i)
    return v / np.linalg.norm(v)


class BlockJacobi:
    """Preconditioner slot: inverse nodal block diagonal of the prepared tangent (src/preconditioners.jl:116)."""


class BlockJacobiState:
    def __init__(self, mf: MatrixFreeJacobian):
        self.mf = mf
        self.nbuild = 0
        self.update(mf)

    def update(self, mf: MatrixFreeJacobian):
        self.mf = mf
        ok = ctypes.c_int()
        call("hfk_blocks_update", mf.op.problem.h, ctypes.byref(ok))
        self.ok = bool(ok.value)
        self.nbuild += 1
        return self

    def ldiv(self, y, r):
        """``ldiv!(y, st, r)`` (src/preconditioners.jl:329-344)."""
        call("hfk_blocks_apply", self.mf.op.problem.h, ptr(r), ptr(y))
        return y

    def blocks(self):
        """(dofs (nb, 3) 1-based, B (nb, 3, 3), Binv (nb, 3, 3))."""
        nb = ctypes.c_int()
        call("hfk_blocks_get", self.mf.op.problem.h, ctypes.byref(nb), None, None, None)
        n = nb.value
        dofs = np.zeros(3 * n, dtype=np.int32)
        B = np.zeros(9 * n)
        Bi = np.zeros(9 * n)
        call("hfk_blocks_get", self.mf.op.problem.h, ctypes.byref(nb), ptr(dofs, np.int32), ptr(B), ptr(Bi))
        return (dofs.reshape(n, 3), B.reshape(n, 3, 3).transpose(0, 2, 1), Bi.reshape(n, 3, 3).transpose(0, 2, 1))


def eigenvalue_bounds(mf: MatrixFreeJacobian, prec: BlockJacobiState, k: int = 10, b=None):
    """``eigenvalue_bounds(mf, prec; k, b)`` (src/preconditioners.jl:374-389): (lmin, lmax)."""
    lo, hi = ctypes.c_double(), ctypes.c_double()
    bb = None if b is None else np.ascontiguousarray(b, dtype=np.float64)
    call("hfk_eigenvalue_bounds", mf.op.problem.h, k, ptr(bb) if bb is not None else None, ctypes.byref(lo),
         ctypes.byref(hi))
    return lo.value, hi.value


def hessenberg_eigvals(H: np.ndarray):
    """Eigenvalues of an upper Hessenberg matrix (the library's host QR iteration)."""
    n = H.shape[0]
    Hf = np.asfortranarray(H, dtype=np.float64)
    re, im = np.zeros(n), np.zeros(n)
    call("hfk_hessenberg_eigvals", n, ptr(Hf), ptr(re), ptr(im))
    return re + 1j * im


class Prolongation:
    """``Prolongation(Uc, Uf)`` (src/transfers.jl:133-154) between two operators' problems on one mesh."""

    def __init__(self, coarse: Problem, fine: Problem):
        Qf, Qc = fine.space.Q, coarse.space.Q
        self.E, self.Einj = transfer_matrices(Qf, Qc)
        h = ctypes.c_void_p()
        call("hfk_transfer_create", ctypes.byref(h), fine.h, coarse.h, ptr(self.E), ptr(self.Einj))
        self.h = h
        self.fine, self.coarse = fine, coarse
        self.nf, self.nc = fine.nfree, coarse.nfree

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            try:
                _lib.lib().hfk_transfer_destroy(h)
            except Exception:
                pass
            self.h = None

    def prolongate(self, yf, xc):
        """``prolongate!(yf, P, xc)`` (src/transfers.jl:238-245)."""
        call("hfk_prolongate", self.h, ptr(xc), ptr(yf))
        return yf

    def restrict(self, yc, yf):
        """``restrict!(yc, P, yf)`` (src/transfers.jl:252-259)."""
        call("hfk_restrict", self.h, ptr(yf), ptr(yc))
        return yc

    def inject(self, xc, dc, xf, df):
        """``inject!(xc, dc, P, xf, df)`` (src/transfers.jl:285-313)."""
        call("hfk_inject", self.h, ptr(xf), ptr(df), ptr(xc), ptr(dc))
        return xc, dc


class PMultigrid:
    """``PMultigrid(spaces; smoother = Chebyshev(), coarse = LUSolver(), coarse_every = 1)`` (src/pmultigrid.jl:256-267).

    ``spaces`` lists the trial spaces of the levels, finest first (same mesh, same closed Dirichlet
    boundary, nested orders). ``coarse`` "cholesky": the coarsest level is assembled and factorised
    on the GPU (dense Cholesky, FP64); "cg": ``coarse_iters`` block-Jacobi CG steps per problem on
    the matrix-free coarsest level (for batches and coarse levels too large for a dense factor; a
    variable preconditioner, use ``krylov="fcg"``). ``precision`` "fp64" or "fp32" (smoothers and
    products of the levels above the coarse one; the eigenvalue estimate and the coarse solve stay
    FP64).
    """

    def __init__(self, spaces, smoother: Chebyshev = Chebyshev(), coarse_every: int = 1, precision: str = "fp64",
                 coarse: str = "cholesky", coarse_iters: int = 20):
        if coarse not in ("cholesky", "cg"):
            raise ValueError("HyperFEMKernels: PMultigrid: coarse must be 'cholesky' or 'cg'")
        if coarse == "cg" and coarse_iters < 1:
            raise ValueError("HyperFEMKernels: PMultigrid: coarse_iters must be ≥ 1")
        self.coarse, self.coarse_iters = coarse, int(coarse_iters)
        if len(spaces) < 2:
            raise ValueError("HyperFEMKernels: PMultigrid needs at least two levels")
        if coarse_every < 1:
            raise ValueError("HyperFEMKernels: PMultigrid: coarse_every must be ≥ 1")
        if precision not in ("fp64", "fp32"):
            raise ValueError("HyperFEMKernels: precision must be 'fp64' or 'fp32'")
        self.spaces = list(spaces)
        self.smoother = smoother
        self.coarse_every = coarse_every
        self.precision = precision


class PMultigridState:
    def __init__(self, prec: PMultigrid, mf: MatrixFreeJacobian):
        self.prec = prec
        op = mf.op
        # level operators captured from the working operator's forms, with the working quadrature
        # (the coarse operators integrate with the fine measure, src/pmultigrid.jl:244-247)
        self.problems = [op.problem]
        for U in prec.spaces[1:]:
            self.problems.append(Problem(U, op.quad, op.res))
        self.P = [Prolongation(self.problems[l + 1], self.problems[l]) for l in range(len(self.problems) - 1)]
        L = len(self.problems)
        lv = (ctypes.c_void_p * L)(*[p.h.value for p in self.problems])
        tr = (ctypes.c_void_p * (L - 1))(*[t.h.value for t in self.P])
        h = ctypes.c_void_p()
        c = prec.smoother
        call("hfk_pmg_create", ctypes.byref(h), L, lv, tr, c.degree, c.range, c.inflate, c.eig_iters, prec.coarse_every,
             _lib.FP32 if prec.precision == "fp32" else _lib.FP64)
        self.h = h
        self._levels = [p.h.value for p in self.problems]
        for hv in self._levels:
            _lib.retain_problem(hv)
        if prec.coarse == "cg":
            call("hfk_pmg_set_coarse", h, _lib.COARSE_CG, prec.coarse_iters)
        if c.eig_inner == "preconditioner":
            call("hfk_pmg_set_eig_inner", h, _lib.EIG_PRECONDITIONED)
        self.ncycle = 0
        self.update(mf)

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            try:
                _lib.lib().hfk_pmg_destroy(h)
                for hv in getattr(self, "_levels", ()):
                    _lib.release_problem(hv)
            except Exception:
                pass
            self.h = None

    def update(self, mf: MatrixFreeJacobian):
        """``preconditioner_update!`` (src/pmultigrid.jl:298-313): levels follow the operator's state."""
        for p in self.problems[1:]:
            p.set_params(mf.op.res)
        ok = ctypes.c_int()
        x = mf.x
        # the levels follow the state the Jacobian was prepared at (its Dirichlet values included)
        d = mf.dvals if mf.dvals is not None else mf.op.dirichlet_values()
        call("hfk_pmg_update", self.h, ptr(x), ptr(d), ctypes.byref(ok))
        self.ok = bool(ok.value)
        return self

    @property
    def nbuild(self) -> int:
        """Coarse builds (assembly and factorisation), the count the reference's
        ``preconditioner_builds`` reports for a p-multigrid (src/pmultigrid.jl:56, :105, :340)."""
        return int(self.stats()["coarse_builds"])

    def ldiv(self, y, r):
        """``ldiv!(y, st, r)`` (src/pmultigrid.jl:331-338): one V-cycle (NaN when not ok)."""
        self.ncycle += 1
        call("hfk_pmg_vcycle", self.h, ptr(r), ptr(y))
        return y

    def stats(self):
        """Counters and times (ms): updates, coarse builds, cycles, update/coarse/blocks/eig/cycle time."""
        out = np.zeros(9)
        call("hfk_pmg_stats", self.h, ptr(out))
        keys = ("updates", "coarse_builds", "cycles", "t_update_ms", "t_coarse_ms", "t_blocks_ms", "t_eig_ms",
                "t_cycle_ms", "t_potrf_ms")
        return dict(zip(keys, out.tolist()))

    def segment_bounds(self, level: int):
        """(lmin, lmax) of the level's eigenvalue estimate per problem of a batch."""
        k = self.problems[level].nseg
        lo, hi = np.zeros(k), np.zeros(k)
        call("hfk_pmg_segment_bounds", self.h, level, ptr(lo), ptr(hi))
        return lo, hi

    def level_info(self, level: int):
        a, b, lo, hi = (ctypes.c_double() for _ in range(4))
        call("hfk_pmg_level_info", self.h, level, ctypes.byref(lo), ctypes.byref(hi), ctypes.byref(a), ctypes.byref(b))
        return dict(lmin=lo.value, lmax=hi.value, a=a.value, b=b.value)


@dataclasses.dataclass
class MatrixFreeSolver:
    """``MatrixFreeSolver(; krylov, rtol, atol, maxiter, restart, preconditioner)`` (src/solvers.jl:33-53).

    ``krylov`` is "gmres" or "fgmres" (restarted, right-preconditioned, ``restart`` iterations per
    cycle as the reference's memory; FGMRES keeps the preconditioned basis and accepts a variable
    preconditioner), "fcg" (flexible CG, for variable preconditioners such as a mixed-precision
    V-cycle) or "cg". The default stays "fcg": the batched solves of ``hfk.batch`` are CG only.
    """

    krylov: str = "fcg"
    rtol: float = 1e-8
    atol: float = 0.0
    maxiter: int = 500
    preconditioner: object = None
    restart: int = 50

    def __post_init__(self):
        if self.krylov not in ("fcg", "cg", "gmres", "fgmres"):
            raise ValueError("HyperFEMKernels: MatrixFreeSolver: krylov must be 'gmres', 'fgmres', 'fcg' or 'cg' "
                             f"(got {self.krylov!r})")
        if self.restart <= 0:
            raise ValueError("HyperFEMKernels: MatrixFreeSolver: restart must be positive")
        if not (0 <= self.rtol < 1):
            raise ValueError(f"HyperFEMKernels: the relative tolerance must be in [0, 1) (got {self.rtol})")
        if self.atol < 0:
            raise ValueError("HyperFEMKernels: MatrixFreeSolver: atol must be ≥ 0")
        if self.maxiter <= 0:
            raise ValueError("HyperFEMKernels: MatrixFreeSolver: maxiter must be positive")


class LaggedAssembled:
    """``LaggedAssembled(solver; every = 3)`` (src/preconditioners.jl:41-97): the operator's tangent
    assembled and factorised at the setup and then every ``every`` updates (a stale factor in
    between). ``solver`` "cholesky": the GPU Cholesky of the assembled tangent, factored and stored
    over the band of the matrix (FP64; memory about 8 n (b + 64) bytes for the lower bandwidth b),
    in place of the reference's Gridap solver."""

    def __init__(self, solver: str = "cholesky", every: int = 3):
        if solver != "cholesky":
            raise ValueError("HyperFEMKernels: LaggedAssembled: solver must be 'cholesky'")
        if every < 1:
            raise ValueError("HyperFEMKernels: LaggedAssembled: every must be ≥ 1")
        self.solver, self.every = solver, int(every)


class SlotState:
    """State of a one-level preconditioner slot (``hfk_slot_create``): ``LaggedAssembled`` or
    ``BlockJacobi`` inside a ``MatrixFreeSolver`` (``preconditioner_setup``/``update!``/``ldiv!``)."""

    def __init__(self, slot, mf: MatrixFreeJacobian):
        if not mf.prepared:
            raise RuntimeError("HyperFEMKernels: the MatrixFreeJacobian has not been prepared")
        kind = _lib.SLOT_BLOCK_JACOBI if isinstance(slot, BlockJacobi) else _lib.SLOT_LAGGED_ASSEMBLED
        # the slot's handle refers to the operator's problem: keep it alive until the slot is gone
        self.problem = mf.op.problem
        h = ctypes.c_void_p()
        call("hfk_slot_create", ctypes.byref(h), mf.op.problem.h, kind, getattr(slot, "every", 1))
        self.h, self.slot = h, slot
        self._levels = [mf.op.problem.h.value]
        _lib.retain_problem(self._levels[0])
        self.update(mf)

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            try:
                _lib.lib().hfk_pmg_destroy(h)
                for hv in getattr(self, "_levels", ()):
                    _lib.release_problem(hv)
            except Exception:
                pass
            self.h = None

    def update(self, mf: MatrixFreeJacobian):
        ok = ctypes.c_int()
        d = mf.dvals if mf.dvals is not None else mf.op.dirichlet_values()
        call("hfk_pmg_update", self.h, ptr(mf.x), ptr(d), ctypes.byref(ok))
        self.ok = bool(ok.value)
        return self

    def ldiv(self, y, r):
        call("hfk_pmg_vcycle", self.h, ptr(r), ptr(y))
        return y

    def stats(self):
        out = np.zeros(9)
        call("hfk_pmg_stats", self.h, ptr(out))
        return {"updates": out[0], "builds": out[1]}

    @property
    def nbuild(self) -> int:
        return int(self.stats()["builds"])


class MatrixFreeSolverNS:
    def __init__(self, solver: MatrixFreeSolver, mf: MatrixFreeJacobian):
        if not mf.prepared:
            raise RuntimeError("HyperFEMKernels: the MatrixFreeJacobian has not been prepared "
                               "(call jacobian!(mf, op, x) before numerical_setup)")
        self.solver, self.mf = solver, mf
        p = solver.preconditioner
        if p is None:
            self.prec = None
        elif isinstance(p, PMultigrid):
            self.prec = PMultigridState(p, mf)
        elif isinstance(p, (LaggedAssembled, BlockJacobi)):
            self.prec = SlotState(p, mf)
        else:
            raise TypeError("HyperFEMKernels: unsupported preconditioner slot")
        self.rtol = solver.rtol
        self.iters, self.converged, self.indefinite, self.rnorm, self.nsetup = 0, True, False, float("nan"), 1

    def update(self, mf):
        self.mf = mf
        self.nsetup += 1
        if self.prec is not None:
            self.prec.update(mf)
        return self


def symbolic_setup(ls: MatrixFreeSolver, mf):
    if not isinstance(mf, MatrixFreeJacobian):
        raise TypeError("HyperFEMKernels: MatrixFreeSolver applies a MatrixFreeJacobian; build the KernelOperator "
                        "with jacobian = 'matrixfree'")
    return ls


def numerical_setup(ss: MatrixFreeSolver, mf: MatrixFreeJacobian) -> MatrixFreeSolverNS:
    return MatrixFreeSolverNS(ss, mf)


def numerical_setup_update(ns: MatrixFreeSolverNS, mf: MatrixFreeJacobian) -> MatrixFreeSolverNS:
    """``numerical_setup!(ns, mf)`` (src/solvers.jl:106-109)."""
    return ns.update(mf)


def solve(x, ns: MatrixFreeSolverNS, b):
    """``solve!(x, ns, b)`` (src/solvers.jl:111-159); x is the initial guess on input."""
    if ns.mf.op.problem.nseg > 1:  # a batch: one solve per problem (hfk.batch)
        from .batch import solve_batched

        solve_batched(x, ns, b)
        return x
    s = ns.solver
    it, conv, ind, rel = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
    prec = ns.prec.h if ns.prec is not None else None
    if s.krylov in ("gmres", "fgmres"):
        call("hfk_solve_gmres", ns.mf.op.problem.h, prec, ptr(b), ptr(x), ns.rtol, s.atol, s.maxiter, s.restart,
             1 if s.krylov == "fgmres" else 0, ctypes.byref(it), ctypes.byref(conv), ctypes.byref(rel))
    else:
        call("hfk_solve_cg", ns.mf.op.problem.h, prec, ptr(b), ptr(x), ns.rtol, s.atol, s.maxiter,
             1 if s.krylov == "fcg" else 0, ctypes.byref(it), ctypes.byref(conv), ctypes.byref(ind), ctypes.byref(rel))
    ns.iters, ns.converged, ns.indefinite, ns.rnorm = it.value, bool(conv.value), bool(ind.value), rel.value
    if prec is not None and s.krylov in ("gmres", "fgmres"):
        # a failed preconditioner: no iteration, indefinite when it met an indefinite tangent
        pok, pind = ctypes.c_int(), ctypes.c_int()
        call("hfk_pmg_status", prec, ctypes.byref(pok), ctypes.byref(pind))
        ns.indefinite = not pok.value and bool(pind.value)
    return x


# hooks read by a Newton solver (src/solvers.jl:164-174)
def linear_converged(ns):
    return ns.converged


def linear_iterations(ns):
    return ns.iters


def linear_indefinite(ns):
    return ns.indefinite


def set_tolerance(ns, rtol):
    if rtol is None:
        ns.rtol = ns.solver.rtol
    else:
        if not (0 <= rtol < 1):
            raise ValueError(f"HyperFEMKernels: the relative tolerance must be in [0, 1) (got {rtol})")
        ns.rtol = float(rtol)
    return ns


def tolerance(ns):
    return ns.rtol


def preconditioner_builds(ns):
    return 0 if ns.prec is None else ns.prec.nbuild
