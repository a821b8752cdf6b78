"""Batched problems: many independent solves advanced by the same kernel launches.

No counterpart in the reference, which solves one problem per operator: here a set of problems
(meshes, materials) becomes one disjoint-union space whose cells and free dofs are laid out
problem after problem ("segments", ``hfk_problem_set_segments``). Every launch (cell kernels,
smoothers, transfers, vector updates) then covers all problems, while what is per problem in the
reference's algorithms stays per problem: the law parameters (per cell), the inner products,
Krylov scalars and stopping tests (``hfk_solve_cg_batched``), the Chebyshev intervals (one
eigenvalue estimate per problem) and the Newton convergence (``newton_solve_batched``).
"""
from __future__ import annotations

import ctypes
import dataclasses
import time

import numpy as np

from . import _lib
from . import solvers as S
from ._lib import call, ptr
from .fespace import CartesianMesh, VectorLagrangeSpace


class _UnionMesh:
    """The cells of all problems, problem after problem: (3, 8, ncells) vertex coordinates."""

    def __init__(self, meshes):
        self.meshes = list(meshes)
        self.coords = np.asfortranarray(np.concatenate([m.coords for m in self.meshes], axis=2))
        self.ncells = int(self.coords.shape[2])


class UnionSpace:
    """Disjoint union of ``VectorLagrangeSpace`` s of one order (one problem each).

    Free dofs, Dirichlet dofs and cells are numbered problem after problem; ``seg_dofs``,
    ``seg_dirs`` and ``seg_cells`` hold the offsets (nseg + 1). ``params`` (nseg x 2) gives lambda,
    mu per problem (None: the forms' parameters everywhere). Duck-types the attributes of a space
    that ``Problem``, ``Prolongation`` and ``PMultigrid`` read.
    """

    def __init__(self, spaces, params=None):
        spaces = list(spaces)
        if not spaces:
            raise ValueError("HyperFEMKernels: a batch needs at least one problem")
        order = spaces[0].order
        if any(s.order != order for s in spaces):
            raise ValueError("HyperFEMKernels: the problems of a batch must have the same order")
        self.spaces = spaces
        self.order, self.Q, self.nn, self.nc, self.ndl = order, spaces[0].Q, spaces[0].nn, 3, spaces[0].ndl
        self.nseg = len(spaces)
        self.seg_dofs = np.concatenate([[0], np.cumsum([s.nfree for s in spaces])]).astype(np.int64)
        self.seg_dirs = np.concatenate([[0], np.cumsum([s.ndir for s in spaces])]).astype(np.int64)
        self.seg_cells = np.concatenate([[0], np.cumsum([s.mesh.ncells for s in spaces])]).astype(np.int32)
        self.nfree, self.ndir = int(self.seg_dofs[-1]), int(self.seg_dirs[-1])
        if self.nfree >= 2**31 or self.seg_cells[-1] >= 2**31:
            raise ValueError("HyperFEMKernels: a batch is limited to 2^31 free dofs and cells")
        self.nnodes = int(sum(s.nnodes for s in spaces))
        self.mesh = _UnionMesh([s.mesh for s in spaces])
        ids = []
        for k, s in enumerate(spaces):
            a = s.cell_dof_ids.astype(np.int64)
            a = np.where(a > 0, a + self.seg_dofs[k], np.where(a < 0, a - self.seg_dirs[k], 0))
            ids.append(a)
        self.cell_dof_ids = np.asfortranarray(np.concatenate(ids, axis=1).astype(np.int32))
        self.dirichlet_values = np.concatenate([s.dirichlet_values for s in spaces])
        self.params = None if params is None else np.ascontiguousarray(np.asarray(params, dtype=float).reshape(self.nseg, 2))

    @property
    def segments(self):
        return self.seg_dofs, self.seg_cells, self.params

    def tables(self, quad):
        return self.spaces[0].tables(quad)

    def split(self, v):
        """Per-problem views of a free-dof vector (numpy or torch)."""
        return [v[self.seg_dofs[k]:self.seg_dofs[k + 1]] for k in range(self.nseg)]

    def split_dirichlet(self, v):
        return [v[self.seg_dirs[k]:self.seg_dirs[k + 1]] for k in range(self.nseg)]


def apply_segments(problem, space):
    """Declare the union's problems to the engine (``hfk_problem_set_segments``)."""
    dofs, cells, params = space.segments
    prm = None if params is None else np.ascontiguousarray(params.ravel())
    call("hfk_problem_set_segments", problem.h, space.nseg, ptr(dofs, np.int64), ptr(cells, np.int32),
         ptr(prm) if prm is not None else None)


def segment_norms(problem, v) -> np.ndarray:
    """||v_s|| for every segment of ``problem``."""
    out = np.zeros(problem.nseg)
    call("hfk_segment_dots", problem.h, ptr(v), ptr(v), ptr(out))
    return np.sqrt(out)


def segment_scale(problem, v, f):
    """v_s *= f[s] (v a CUDA tensor)."""
    f = np.ascontiguousarray(f, dtype=float)
    call("hfk_segment_scale", problem.h, ptr(v), ptr(f))
    return v


@dataclasses.dataclass
class BatchedSolveResult:
    iters: np.ndarray
    converged: np.ndarray
    indefinite: np.ndarray
    relres: np.ndarray
    sweeps: int


def solve_batched(x, ns: S.MatrixFreeSolverNS, b) -> BatchedSolveResult:
    """``solve!`` on every problem of a batched operator (``hfk_solve_cg_batched``)."""
    s = ns.solver
    if s.krylov not in ("cg", "fcg"):
        raise ValueError("HyperFEMKernels: batched solves run CG or FCG (krylov = 'cg' or 'fcg')")
    p = ns.mf.op.problem
    k = p.nseg
    it = np.zeros(k, dtype=np.int32)
    conv = np.zeros(k, dtype=np.int32)
    ind = np.zeros(k, dtype=np.int32)
    rel = np.zeros(k)
    sw = ctypes.c_int()
    prec = ns.prec.h if ns.prec is not None else None
    call("hfk_solve_cg_batched", p.h, prec, ptr(b), ptr(x), ns.rtol, s.atol, s.maxiter, 1 if s.krylov == "fcg" else 0,
         ptr(it, np.int32), ptr(conv, np.int32), ptr(ind, np.int32), ptr(rel), ctypes.byref(sw))
    res = BatchedSolveResult(it, conv.astype(bool), ind.astype(bool), rel, sw.value)
    ns.iters, ns.converged, ns.indefinite = int(it.max(initial=0)), bool(res.converged.all()), bool(res.indefinite.any())
    ns.rnorm = float(rel.max(initial=0.0))
    ns.batched = res
    return res


@dataclasses.dataclass
class BatchedNewtonStats:
    load_steps: int = 0
    newton_sweeps: int = 0                      # Newton iterations of the common loop
    krylov_sweeps: list = dataclasses.field(default_factory=list)  # common Krylov loop lengths
    newton_iters: np.ndarray = None             # per problem
    krylov_iters: np.ndarray = None             # per problem, summed over its Newton steps
    residual_norms: list = dataclasses.field(default_factory=list)  # per sweep: (nseg,) norms
    converged: np.ndarray = None                # per problem
    seconds: float = 0.0
    pmg: dict = None


def newton_solve_batched(op, solver: S.MatrixFreeSolver, g_full: np.ndarray, loads, x0=None, *, rtol_newton=1e-8,
                         atol_newton=1e-12, max_newton=20, lift=None, on_setup=None):
    """Newton with load stepping on every problem of a batched operator at once.

    The per-problem algorithm is the one of ``newton_solve`` (the reference's Newton loop,
    ``test/solvers/test_pmultigrid.jl:86-115``): per problem, Newton stops when
    ||R_s|| <= max(rtol_newton ||R_s,0||, atol_newton). Problems that have converged get a zero
    right-hand side (their Krylov solve stops at once) while the others continue.
    ``lift`` (free dofs, at load factor 1): a field that carries the Dirichlet data into the
    interior; each load step starts from x + (load increment) * lift instead of x, which keeps the
    first iterate of a step free of a strain jump at the loaded boundary (``newton_solve``'s
    ``lift``). ``on_setup(ns)`` is called once the solver's numerical set-up exists.
    """
    import torch

    U = op.U
    p = op.problem
    k = U.nseg
    n = U.nfree
    dev = torch.device("cuda")
    x = torch.zeros(n, dtype=torch.float64, device=dev) if x0 is None else torch.as_tensor(x0, device=dev).clone()
    b = torch.zeros(n, dtype=torch.float64, device=dev)
    dx = torch.zeros(n, dtype=torch.float64, device=dev)
    mf = op.allocate_jacobian(x)
    ns = None
    st = BatchedNewtonStats(newton_iters=np.zeros(k, dtype=np.int64), krylov_iters=np.zeros(k, dtype=np.int64),
                            converged=np.ones(k, dtype=bool))
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
            rn = segment_norms(p, b)
            st.residual_norms.append(rn)
            if r0 is None:
                r0 = rn.copy()
            active = rn > np.maximum(rtol_newton * r0, atol_newton)
            if not active.any():
                break
            mf.prepare(x, dv)
            if ns is None:
                ns = S.numerical_setup(S.symbolic_setup(solver, mf), mf)
                if on_setup is not None:
                    on_setup(ns)
            else:
                S.numerical_setup_update(ns, mf)
            dx.zero_()
            b.neg_()
            segment_scale(p, b, active.astype(float))
            res = solve_batched(dx, ns, b)
            st.krylov_sweeps.append(res.sweeps)
            st.krylov_iters += res.iters
            st.newton_iters += active
            st.newton_sweeps += 1
            failed = active & ~res.converged
            if failed.any():
                st.converged &= ~failed
                break
            x += dx
        else:
            st.converged &= ~active
        if not st.converged.all():
            break
    torch.cuda.synchronize()
    st.seconds = time.perf_counter() - t0
    if ns is not None and ns.prec is not None and hasattr(ns.prec, "stats"):
        st.pmg = ns.prec.stats()
    return x, st


def shard_problems(problems, rank: int, world: int):
    """Indices of the problems rank ``rank`` of ``world`` solves: independent problems shard with no
    exchange; greedy balance of the free-dof counts (largest first onto the least loaded rank),
    deterministic, so every rank computes the same partition without communicating."""
    cost = [3 * (2 * q.n + 1) ** 3 for q in problems]
    load = [0] * world
    owner = [0] * len(problems)
    for k in sorted(range(len(problems)), key=lambda k: (-cost[k], k)):
        r = min(range(world), key=lambda r: (load[r], r))
        owner[k] = r
        load[r] += cost[k]
    return [k for k in range(len(problems)) if owner[k] == rank]


@dataclasses.dataclass(frozen=True)
class BatchProblem:
    n: int          # cells per direction
    lam: float
    mu: float


def draw_batch(count=256, nmin=8, nmax=24, lam_range=(0.5, 20.0), mu_range=(0.2, 5.0), seed=4):
    """``count`` problems: cells per direction uniform in {nmin..nmax}, (lambda, mu) log-uniform."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(nmin, nmax + 1, size=count)
    lam = np.exp(rng.uniform(np.log(lam_range[0]), np.log(lam_range[1]), size=count))
    mu = np.exp(rng.uniform(np.log(mu_range[0]), np.log(mu_range[1]), size=count))
    return [BatchProblem(int(a), float(b), float(c)) for a, b, c in zip(ns, lam, mu)]


def cube_lifting(union, displacement=0.05):
    """Free-dof values of u = displacement * x e_x on every problem of ``union`` (the affine field
    that matches ``cube_batch``'s Dirichlet data at load factor 1)."""
    f = lambda X: np.column_stack([displacement * X[:, 0], 0 * X[:, 1], 0 * X[:, 2]])
    return np.concatenate([V.interpolate(f)[0] for V in union.spaces])


def cube_batch(problems, orders=(2, 1), displacement=0.05):
    """Union spaces (finest order first) of unit cubes n^3, x = 0 clamped, x = 1 moved by
    ``displacement`` along x; returns (union spaces, Dirichlet values at load factor 1)."""
    g = (lambda X: np.zeros_like(X), lambda X: np.column_stack([np.full(len(X), displacement), 0 * X[:, 1], 0 * X[:, 2]]))
    params = np.array([[q.lam, q.mu] for q in problems])
    unions = []
    for order in orders:
        spaces = [VectorLagrangeSpace(CartesianMesh((q.n, q.n, q.n)), order, dirichlet=("x0", "x1"), g=g)
                  for q in problems]
        unions.append(UnionSpace(spaces, params))
    return unions, unions[0].dirichlet_values.copy()
