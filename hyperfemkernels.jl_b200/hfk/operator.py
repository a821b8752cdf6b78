"""``KernelOperator`` and ``MatrixFreeJacobian`` over the B200 engine.

Mirrors the reference's operator API (HyperFEMKernels ``src/assembly.jl:630-666``, ``:904-933``,
``src/matrixfree.jl:33-260``): the same method names (without Julia's ``!``; in-place methods
write into their first argument and return it), the same argument meaning and the same error
prefix. Every numerical call goes through ``libhfk.so``; there is no CPU path.
"""
from __future__ import annotations

import ctypes

import numpy as np
import scipy.sparse as sp

from . import _lib
from ._lib import call, ptr
from .fespace import Quadrature, VectorLagrangeSpace, geometry_tables
from .forms import Form


class Problem:
    """One device-resident group: tables, geometry, ids, colours (``hfk_problem``)."""

    def __init__(self, space: VectorLagrangeSpace, quad: Quadrature, form: Form):
        self.space, self.quad = space, quad
        Nt, dNt = space.tables(quad)
        dMt = geometry_tables(quad.points())
        self._keep = (Nt, dNt, dMt)
        prm = np.array(form.params(), dtype=np.float64)
        h = ctypes.c_void_p()
        call("hfk_problem_create", ctypes.byref(h), space.nn, quad.np, 8, space.mesh.ncells, ptr(quad.xq), ptr(quad.w),
             ptr(Nt), ptr(dNt), ptr(dMt), ptr(space.mesh.coords), ptr(space.cell_dof_ids, np.int32), space.nfree,
             space.ndir, form.law, ptr(prm), len(prm))
        self.h = h
        self.nfree, self.ndir = space.nfree, space.ndir
        self.form = form
        self.nseg = 1
        if getattr(space, "segments", None) is not None:
            from .batch import apply_segments  # a union of independent problems

            apply_segments(self, space)
            self.nseg = space.nseg

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            try:
                _lib.destroy_problem(h.value)  # deferred while a hierarchy still uses it
            except Exception:
                pass
            self.h = None

    def info(self):
        nfree, nnz = ctypes.c_int64(), ctypes.c_int64()
        Q, P, nc = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        call("hfk_problem_info", self.h, ctypes.byref(nfree), ctypes.byref(Q), ctypes.byref(P), ctypes.byref(nc),
             ctypes.byref(nnz))
        return dict(nfree=nfree.value, Q=Q.value, P=P.value, ncolors=nc.value, nnz=nnz.value)

    def set_params(self, form: Form):
        prm = np.array(form.params(), dtype=np.float64)
        call("hfk_problem_set_params", self.h, ptr(prm), len(prm))
        self.form = form

    def set_stream(self, stream_handle: int | None):
        call("hfk_problem_set_stream", self.h, ctypes.c_void_p(stream_handle or 0))

    def set_scatter(self, mode: str):
        """"auto" (default), "coloured" (deterministic) or "atomic" for the sum-factorised kernels and
        the restriction from this level."""
        m = {"auto": _lib.SCATTER_AUTO, "coloured": _lib.SCATTER_COLOURED, "atomic": _lib.SCATTER_ATOMIC}[mode]
        call("hfk_problem_set_scatter", self.h, m)

    def set_launch(self, kernel: str = "line", warps: int = 4):
        """Launch shape under an explicit scatter mode: "line" (the line-mapped kernels, 2 or 4 warps
        per CTA), "point" (the point-parallel matrix-free product, warps 0 = one cell per CTA or
        8), "tensor" (the FP32 product of Q2 cells with both contractions on the tensor cores) or
        "q1" (the warp-synchronous product of Q1 cells with 2^3 points); with the last two the other
        kernels take the line-mapped shape of 4 warps."""
        call("hfk_problem_set_launch", self.h, {"line": 0, "point": 1, "tensor": 2, "q1": 3}[kernel], int(warps))

    def set_assembly_kernel(self, kernel: str = "fma"):
        """Kernel of the assembled Jacobian on 27-node cells: "fma" (default: the element blocks of the
        symmetric tangent on the FP64 FMA pipe) or "tensor" (on the FP64 tensor cores)."""
        call("hfk_problem_set_assembly_kernel", self.h, {"fma": 0, "tensor": 1}[kernel])

    def set_solve_graph(self, on: bool = True):
        """Batched CG on this operator: the iterations after the second as one CUDA graph launch that
        loops on the device (default), or the host-driven loop."""
        call("hfk_problem_set_solve_graph", self.h, 1 if on else 0)

    def tuning(self, kernel: str = "jv", precision: str = "fp64"):
        """The launch-shape autotuner's choice: {"atomic": bool, "kernel": "line" | "point",
        "warps": int} or None (not run yet)."""
        a, k, w = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        call("hfk_problem_tuning", self.h, {"jv": 0, "residual": 1, "jv_stored": 2}[kernel],
             _lib.FP32 if precision == "fp32" else _lib.FP64, ctypes.byref(a), ctypes.byref(k), ctypes.byref(w))
        return None if a.value < 0 else {"atomic": bool(a.value), "kernel": ("line", "point", "tensor", "q1")[k.value],
                                         "warps": w.value}

    def launches(self) -> int:
        c = ctypes.c_int64()
        call("hfk_launch_count", self.h, ctypes.byref(c))
        return c.value

    def device_errors(self) -> int:
        """Bounded device waits of this problem's kernels that ran out since the last call
        (``hfk_problem_device_errors``; 0 in a healthy run)."""
        e = ctypes.c_int()
        call("hfk_problem_device_errors", self.h, ctypes.byref(e))
        return e.value

    def set_timing(self, on: bool = True):
        """Bracket every element-kernel launch sequence with CUDA events (``hfk_problem_set_timing``)."""
        call("hfk_problem_set_timing", self.h, int(bool(on)))

    def kernel_time(self):
        """(summed milliseconds, number of sequences) of the bracketed element-kernel launches since
        timing was switched on or last read (``hfk_problem_kernel_time``)."""
        ms, n = ctypes.c_double(), ctypes.c_int64()
        call("hfk_problem_kernel_time", self.h, ctypes.byref(ms), ctypes.byref(n))
        return ms.value, n.value

    def colors(self) -> np.ndarray:
        out = np.zeros(self.space.mesh.ncells, dtype=np.int32)
        call("hfk_colors", self.h, ptr(out, np.int32))
        return out


class KernelOperator:
    """``KernelOperator(res, jac, U, V; jacobian = :assembled | :matrixfree)`` (``src/assembly.jl:630-666``).

    ``res``/``jac`` are recognised forms (``hfk.forms``); ``U``/``V`` the trial and test spaces
    (same numbering). Not reentrant, like the reference (``src/assembly.jl:363-367``).
    """

    def __init__(self, res: Form, jac: Form, U: VectorLagrangeSpace, V: VectorLagrangeSpace | None = None, *,
                 jacobian: str = "assembled", problem: Problem | None = None):
        if jacobian not in ("assembled", "matrixfree"):
            raise ValueError("HyperFEMKernels: jacobian must be 'assembled' or 'matrixfree'")
        if not res.same_law(jac):
            raise ValueError("HyperFEMKernels: the residual and Jacobian forms are of different laws or measures")
        V = U if V is None else V
        if V.nfree != U.nfree or V.cell_dof_ids is not U.cell_dof_ids and not np.array_equal(V.cell_dof_ids, U.cell_dof_ids):
            raise ValueError("HyperFEMKernels: test and trial spaces with different numbering are not supported")
        self.res, self.jac, self.U, self.V = res, jac, U, V
        self.jacobian_kind = jacobian
        self.quad = Quadrature.gauss(res.degree)
        self.problem = problem if problem is not None else Problem(U, self.quad, res)
        self._pattern = None
        self._checked = []

    # --- Algebra interface (src/assembly.jl:904-933) ---------------------------------------
    def allocate_residual(self, x=None):
        return np.zeros(self.V.nfree)

    def zero_initial_guess(self):
        return np.zeros(self.U.nfree)

    def sparsity_pattern(self) -> sp.csc_matrix:
        """``sparsity_pattern(op)`` (src/assembly.jl:768): the CSC pattern with structural zeros."""
        if self._pattern is None:
            nnz = ctypes.c_int64()
            call("hfk_pattern_build", self.problem.h, ctypes.byref(nnz))
            colptr = np.zeros(self.U.nfree + 1, dtype=np.int64)
            rowval = np.zeros(nnz.value, dtype=np.int64)
            call("hfk_pattern_get", self.problem.h, ptr(colptr, np.int64), ptr(rowval, np.int64))
            A0 = sp.csc_matrix((np.zeros(nnz.value), rowval - 1, colptr - 1), shape=(self.V.nfree, self.U.nfree))
            self._pattern = (A0, colptr, rowval)
        return self._pattern[0]

    def pattern_julia(self):
        """(colptr, rowval) 1-based, as Julia's SparseMatrixCSC stores them."""
        self.sparsity_pattern()
        return self._pattern[1], self._pattern[2]

    def nonzero_positions(self) -> np.ndarray:
        """``nonzero_positions(op)`` (src/assembly.jl:771): (ndl*ndl, ncells) Int32, 1-based."""
        self.sparsity_pattern()
        ndl, nc = self.U.ndl, self.U.mesh.ncells
        out = np.zeros((ndl * ndl, nc), dtype=np.int32, order="F")
        call("hfk_nonzero_positions", self.problem.h, ptr(out, np.int32))
        return out

    def allocate_jacobian(self, x=None):
        if self.jacobian_kind == "matrixfree":
            return MatrixFreeJacobian(self)
        A = self.sparsity_pattern().copy()
        self._checked.append(id(A.indptr))
        return A

    def _check_matrix(self, A):
        A0 = self.sparsity_pattern()
        if A.shape != A0.shape or A.nnz != A0.nnz:
            raise ValueError(f"HyperFEMKernels: the matrix ({A.shape}, {A.nnz} nonzeros) does not have the sparsity "
                             f"pattern of the operator ({A0.shape}, {A0.nnz})")
        if id(A.indptr) in self._checked:
            return
        if not (np.array_equal(A.indptr, A0.indptr) and np.array_equal(A.indices, A0.indices)):
            raise ValueError("HyperFEMKernels: the matrix does not have the sparsity pattern of the operator")
        self._checked.append(id(A.indptr))

    def dirichlet_values(self):
        return np.ascontiguousarray(self.U.dirichlet_values, dtype=np.float64)

    def functional(self, x, dvals=None, kind: str = "energy") -> float:
        """``KernelFunctional`` of the operator's law (src/functionals.jl:10-27): "energy" (the
        stored energy Σ Ψ dV, reduce = :sum) or "min_detF" (min over the points, reduce = :min)."""
        d = self.dirichlet_values() if dvals is None else dvals
        out = ctypes.c_double()
        call("hfk_functional", self.problem.h, ptr(x), ptr(d), {"energy": 0, "min_detF": 1}[kind], ctypes.byref(out))
        return out.value

    def residual(self, b, x, dvals=None):
        """``residual!(b, op, x)`` (src/assembly.jl:909-916); Dirichlet values re-read from ``U``."""
        d = self.dirichlet_values() if dvals is None else dvals
        call("hfk_residual", self.problem.h, ptr(x), ptr(d), ptr(b))
        return b

    def jacobian_values(self, nzval, x, dvals=None):
        """The nonzeros of ``jacobian!`` into a vector (host or device) in ``rowval`` order."""
        self.sparsity_pattern()
        d = self.dirichlet_values() if dvals is None else dvals
        call("hfk_jacobian", self.problem.h, ptr(x), ptr(d), ptr(nzval))
        return nzval

    def jacobian(self, A, x):
        """``jacobian!(A, op, x)`` (src/assembly.jl:918-927) or ``jacobian!(mf, op, x)`` (prepare)."""
        if isinstance(A, MatrixFreeJacobian):
            A.rebind(self)
            return A.prepare(x)
        self._check_matrix(A)
        data = np.zeros(A.nnz)
        self.jacobian_values(data, x)
        A.data[:] = data
        return A

    def residual_and_jacobian(self, b, A, x):
        self.residual(b, x)
        self.jacobian(A, x)
        return b, A

    def update(self, res: Form, jac: Form) -> "KernelOperator":
        """``update(op, res, jac)`` (src/assembly.jl:693-744): same structure, new parameters; tables,
        pattern and colours are kept."""
        if not res.same_law(jac):
            raise ValueError("HyperFEMKernels: the residual and Jacobian forms are of different laws or measures")
        if res.law != self.res.law or res.degree != self.res.degree:
            return KernelOperator(res, jac, self.U, self.V, jacobian=self.jacobian_kind)
        self.problem.set_params(res)
        new = KernelOperator.__new__(KernelOperator)
        new.__dict__.update(self.__dict__)
        new.res, new.jac = res, jac
        return new


class MatrixFreeJacobian:
    """``MatrixFreeJacobian(op)`` (src/matrixfree.jl:33-72): ``prepare`` at a state, then ``mul``.

    ``mode`` is ``"recompute"`` (the tangent is re-evaluated inside every product from the state;
    no per-point storage) or ``"stored"`` (the reference's partial assembly: T, inv(Jt), dV per point).
    """

    def __init__(self, op: KernelOperator, mode: str = "recompute"):
        if mode not in ("recompute", "stored"):
            raise ValueError("HyperFEMKernels: mode must be 'recompute' or 'stored'")
        self.op = op
        self.mode = mode
        self.x = np.zeros(0)
        self.dvals = None
        self.prepared = False

    @property
    def shape(self):
        return (self.op.V.nfree, self.op.U.nfree)

    def size(self, i=None):
        return self.shape if i is None else self.shape[i - 1]

    def rebind(self, op: KernelOperator):
        if op is self.op:
            return self
        if (op.V.nfree, op.U.nfree) != self.shape:
            raise ValueError("HyperFEMKernels: the MatrixFreeJacobian was built for an operator on other FE spaces")
        self.op = op
        return self

    def prepare(self, x, dvals=None):
        """``prepare!(mf, x)`` (src/matrixfree.jl:140-159)."""
        d = self.op.dirichlet_values() if dvals is None else dvals
        mode = _lib.MF_STORED if self.mode == "stored" else _lib.MF_RECOMPUTE
        call("hfk_mf_prepare", self.op.problem.h, ptr(x), ptr(d), mode)
        self.x = x.copy() if isinstance(x, np.ndarray) else x.clone()
        # the Dirichlet values of the prepared state (the p-multigrid levels follow this state)
        self.dvals = d.copy() if isinstance(d, np.ndarray) else d.clone()
        self.prepared = True
        return self

    def mul(self, y, dx):
        """``mul!(y, mf, dx)`` (src/matrixfree.jl:246-260)."""
        if not self.prepared:
            raise RuntimeError("HyperFEMKernels: the MatrixFreeJacobian has not been prepared")
        call("hfk_mf_apply", self.op.problem.h, ptr(dx), ptr(y))
        return y

    def mul_many(self, ys, dxs):
        """``mul!`` over a list of vectors in one call: the host copies of one vector overlap the
        product of the next (page-locked host buffers), device vectors are used in place."""
        if not self.prepared:
            raise RuntimeError("HyperFEMKernels: the MatrixFreeJacobian has not been prepared")
        if len(ys) != len(dxs):
            raise ValueError("HyperFEMKernels: as many outputs as inputs")
        k = len(dxs)
        pin = (ctypes.c_void_p * max(k, 1))(*[ptr(a).value for a in dxs])
        pout = (ctypes.c_void_p * max(k, 1))(*[ptr(a).value for a in ys])
        call("hfk_mf_apply_many", self.op.problem.h, k, ctypes.cast(pin, ctypes.c_void_p),
             ctypes.cast(pout, ctypes.c_void_p))
        return ys

    def mul_f32(self, y, dx):
        """The same product in FP32 (mixed-precision smoothers)."""
        call("hfk_mf_apply_f32", self.op.problem.h, ptr(dx, np.float32), ptr(y, np.float32))
        return y

    def __matmul__(self, dx):
        y = np.zeros(self.shape[0])
        return self.mul(y, np.ascontiguousarray(dx, dtype=np.float64))
