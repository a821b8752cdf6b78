"""Python binding and solver driver of the CPU oracle.

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline, never by the product. The element-level kernels are C++/OpenMP (``hfk_oracle.cpp``);
the solver level (Chebyshev smoother, Arnoldi eigenvalue bounds, V-cycle, CG, LU coarse solve)
is restated here with numpy/scipy, as the reference orchestrates it from Julia with Krylov.jl,
LAPACK and Gridap's LUSolver.

Parity status: unpinned against the reference itself (Julia/Gridap cannot run here and the
reference ships no golden vectors); pinned by the reference's known-answer and property tests,
restated in tests/test_oracle.py.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

c_dp = ctypes.POINTER(ctypes.c_double)
c_ip = ctypes.POINTER(ctypes.c_int32)
c_lp = ctypes.POINTER(ctypes.c_int64)


def build():
    """Compile ``libhfk_oracle.so`` next to this file."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libhfk_oracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.o_create.restype = ctypes.c_void_p
        L.o_create.argtypes = [ctypes.c_int] * 4 + [c_dp] * 6 + [c_ip, ctypes.c_int64, ctypes.c_int64,
                                                                   ctypes.c_int, c_dp, ctypes.c_int]
        L.o_free.argtypes = [ctypes.c_void_p]
        L.o_has_tp.argtypes = [ctypes.c_void_p]
        L.o_affine_count.argtypes = [ctypes.c_void_p]
        L.o_set_params.argtypes = [ctypes.c_void_p, c_dp, ctypes.c_int]
        L.o_color.argtypes = [ctypes.c_void_p, c_ip]
        L.o_pattern.restype = ctypes.c_int64
        L.o_pattern.argtypes = [ctypes.c_void_p]
        L.o_pattern_get.argtypes = [ctypes.c_void_p, c_lp, c_lp, c_ip]
        L.o_element_residual.argtypes = [ctypes.c_void_p, c_dp, c_dp, ctypes.c_int, c_dp]
        L.o_element_jacobian.argtypes = [ctypes.c_void_p, c_dp, c_dp, ctypes.c_int, ctypes.c_int, c_dp]
        L.o_residual.argtypes = [ctypes.c_void_p, c_dp, c_dp, c_dp, ctypes.c_int]
        L.o_jacobian.argtypes = [ctypes.c_void_p, c_dp, c_dp, c_dp, ctypes.c_int, ctypes.c_int]
        L.o_mf_prepare.argtypes = [ctypes.c_void_p, c_dp, c_dp, ctypes.c_int]
        L.o_mf_get.argtypes = [ctypes.c_void_p, c_dp, c_dp, c_dp]
        L.o_mf_apply.argtypes = [ctypes.c_void_p, c_dp, c_dp, ctypes.c_int]
        L.o_blocks.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.o_blocks_get.argtypes = [ctypes.c_void_p, c_ip, c_dp, c_dp]
        L.o_blocks_apply.argtypes = [ctypes.c_void_p, c_dp, c_dp]
        L.o_point_law.argtypes = [ctypes.c_int, c_dp, c_dp, c_dp, c_dp]
        L.o_transfer_create.restype = ctypes.c_void_p
        L.o_transfer_create.argtypes = [ctypes.c_int] * 3 + [c_dp, c_dp, c_ip, c_ip, ctypes.c_int64, ctypes.c_int64]
        L.o_transfer_free.argtypes = [ctypes.c_void_p]
        L.o_prolongate.argtypes = [ctypes.c_void_p, c_dp, c_dp]
        L.o_restrict.argtypes = [ctypes.c_void_p, c_dp, c_dp]
        L.o_inject.argtypes = [ctypes.c_void_p, c_dp, c_dp, c_dp, c_dp]
        L.o_functional.restype = ctypes.c_double
        L.o_functional.argtypes = [ctypes.c_void_p, c_dp, c_dp, ctypes.c_int]
        L.o_oseen_create.restype = ctypes.c_void_p
        L.o_oseen_create.argtypes = [ctypes.c_int, ctypes.c_int] + [c_dp] * 7 + [c_ip, ctypes.c_int64, ctypes.c_int64,
                                                                                  c_dp]
        L.o_oseen_free.argtypes = [ctypes.c_void_p]
        L.o_oseen_set_history.argtypes = [ctypes.c_void_p, c_dp, c_dp, c_dp, c_dp]
        L.o_oseen_element.argtypes = [ctypes.c_void_p, ctypes.c_int, c_dp, c_dp]
        L.o_oseen_pattern.restype = ctypes.c_int64
        L.o_oseen_pattern.argtypes = [ctypes.c_void_p]
        L.o_oseen_pattern_get.argtypes = [ctypes.c_void_p, c_lp, c_lp, c_ip]
        L.o_oseen_residual.argtypes = [ctypes.c_void_p, c_dp, c_dp, c_dp, ctypes.c_int]
        L.o_oseen_jacobian.argtypes = [ctypes.c_void_p, c_dp, ctypes.c_int]
        L.o_oseen_set_outlet.argtypes = [ctypes.c_void_p, ctypes.c_int, c_ip, c_ip, c_dp, c_dp, ctypes.c_int, c_dp, c_dp,
                                         ctypes.c_double, ctypes.c_double]
        _LIB = L
    return _LIB


def _d(a):
    if a is None:
        return ctypes.cast(0, c_dp)
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.flags.c_contiguous), a.dtype
    return a.ctypes.data_as(c_dp)


def _i(a):
    if a is None:
        return ctypes.cast(0, c_ip)
    assert a.dtype == np.int32
    return a.ctypes.data_as(c_ip)


def _l(a):
    if a is None:
        return ctypes.cast(0, c_lp)
    assert a.dtype == np.int64
    return a.ctypes.data_as(c_lp)


LAW_SVK = 1
LAW_LINEAR = 2


def point_law(law, params, F):
    """(P, T) of a law at one deformation gradient F (3x3), slot s = c*3 + J."""
    Fc = np.asfortranarray(np.asarray(F, dtype=float))
    P = np.zeros((3, 3), order="F")
    T = np.zeros((9, 9), order="F")
    prm = np.asarray(params, dtype=float)
    lib().o_point_law(law, _d(prm), _d(Fc), _d(P), _d(T))
    return P, T


class OracleProblem:
    """One volume group of a vector Lagrangian field (the reference's ``Group`` + its ``FieldLayout``)."""

    def __init__(self, space, quad, law=LAW_SVK, params=(2.0, 1.0)):
        from hfk.fespace import geometry_tables  # host module (pure numpy)

        self.space = space
        self.quad = quad
        self.Nt, self.dNt = space.tables(quad)
        self.dMt = geometry_tables(quad.points())
        self.params = np.array(list(params) + [0.0] * (5 - len(params)), dtype=float)
        self.ids = space.cell_dof_ids
        self.ncells = space.mesh.ncells
        self.nfree, self.ndir = space.nfree, space.ndir
        self.ndl = space.ndl
        L = lib()
        self.h = L.o_create(self.ncells, space.nn, quad.np, 8, _d(quad.xq), _d(quad.w), _d(self.Nt), _d(self.dNt),
                            _d(self.dMt), _d(space.mesh.coords), _i(self.ids), self.nfree, self.ndir, law,
                            _d(self.params), len(self.params))
        self.colors = np.zeros(self.ncells, dtype=np.int32)
        self.ncolors = L.o_color(self.h, _i(self.colors))
        if self.ncolors < 0:
            raise RuntimeError("HyperFEMKernels: more than 128 colours needed")
        self.nnz = None
        self.prepared = False
        self.nblocks = None

    def __del__(self):
        if getattr(self, "h", None):
            lib().o_free(self.h)
            self.h = None

    def set_params(self, params):
        self.params = np.array(list(params) + [0.0] * (5 - len(params)), dtype=float)
        lib().o_set_params(self.h, _d(self.params), len(self.params))

    @property
    def has_tp(self):
        return bool(lib().o_has_tp(self.h))

    def pattern(self):
        if self.nnz is None:
            self.nnz = int(lib().o_pattern(self.h))
            self.colptr = np.zeros(self.nfree + 1, dtype=np.int64)
            self.rowval = np.zeros(self.nnz, dtype=np.int64)
            self.nzpos = np.zeros((self.ndl * self.ndl, self.ncells), dtype=np.int32, order="F")
            lib().o_pattern_get(self.h, _l(self.colptr), _l(self.rowval), _i(self.nzpos))
        return self.colptr, self.rowval

    def residual(self, x, dvals, nthreads=0):
        b = np.zeros(self.nfree)
        lib().o_residual(self.h, _d(np.ascontiguousarray(x, float)), _d(np.ascontiguousarray(dvals, float)), _d(b), nthreads)
        return b

    def jacobian_values(self, x, dvals, nthreads=0, point_block=12, out=None):
        """The CSC values of jacobian! (the restatement zero-fills them first); ``out``: a float64
        array of nnz entries to assemble into in place, as jacobian!(A, ...) does into A."""
        self.pattern()
        nz = np.zeros(self.nnz) if out is None else out
        assert nz.dtype == np.float64 and nz.size == self.nnz and nz.flags.c_contiguous
        lib().o_jacobian(self.h, _d(np.ascontiguousarray(x, float)), _d(np.ascontiguousarray(dvals, float)), _d(nz),
                         nthreads, point_block)
        return nz

    def jacobian(self, x, dvals, nthreads=0):
        nz = self.jacobian_values(x, dvals, nthreads)
        return sp.csc_matrix((nz, self.rowval - 1, self.colptr - 1), shape=(self.nfree, self.nfree))

    def element_residual(self, x, dvals, cell):
        re = np.zeros(self.ndl)
        lib().o_element_residual(self.h, _d(np.ascontiguousarray(x, float)), _d(np.ascontiguousarray(dvals, float)),
                                 cell, _d(re))
        return re

    def element_jacobian(self, x, dvals, cell, point_block=12):
        KeT = np.zeros((self.ndl, self.ndl), order="F")
        lib().o_element_jacobian(self.h, _d(np.ascontiguousarray(x, float)), _d(np.ascontiguousarray(dvals, float)),
                                 cell, point_block, _d(KeT))
        return KeT

    def functional(self, x, dvals, kind="energy"):
        """KernelFunctional restatement: "energy" (Σ Ψ dV) or "min_detF" (min over the points)."""
        return float(lib().o_functional(self.h, _d(np.ascontiguousarray(x, float)), _d(np.ascontiguousarray(dvals, float)),
                                        {"energy": 0, "min_detF": 1}[kind]))

    def mf_prepare(self, x, dvals, nthreads=0):
        lib().o_mf_prepare(self.h, _d(np.ascontiguousarray(x, float)), _d(np.ascontiguousarray(dvals, float)), nthreads)
        self.prepared = True

    def mf_data(self):
        npq = self.quad.np * self.ncells
        T = np.zeros(81 * npq)
        iJt = np.zeros(9 * npq)
        dV = np.zeros(npq)
        lib().o_mf_get(self.h, _d(T), _d(iJt), _d(dV))
        return T, iJt, dV

    def mf_apply(self, dx, nthreads=0, out=None):
        """y = J dx (the restatement zero-fills y first); ``out``: a float64 array of nfree entries
        to write in place, as mul!(y, J, dx) does."""
        y = np.zeros(self.nfree) if out is None else out
        assert y.dtype == np.float64 and y.size == self.nfree and y.flags.c_contiguous
        rc = lib().o_mf_apply(self.h, _d(np.ascontiguousarray(dx, float)), _d(y), nthreads)
        if rc != 0:
            raise RuntimeError("oracle: mf_apply needs a tensor-product table and prepare()")
        return y

    def blocks(self):
        nb = lib().o_blocks(self.h, 0)
        if nb < 0:
            raise RuntimeError("oracle: blocks need prepare()")
        self.nblocks = nb
        dofs = np.zeros(3 * nb, dtype=np.int32)
        B = np.zeros(9 * nb)
        Binv = np.zeros(9 * nb)
        lib().o_blocks_get(self.h, _i(dofs), _d(B), _d(Binv))
        return dofs.reshape(nb, 3), B.reshape(nb, 3, 3).transpose(0, 2, 1), Binv.reshape(nb, 3, 3).transpose(0, 2, 1)

    def blocks_apply(self, r):
        y = np.zeros(self.nfree)
        lib().o_blocks_apply(self.h, _d(np.ascontiguousarray(r, float)), _d(y))
        return y


class OracleTransfer:
    """``Prolongation`` between two levels on the same mesh (``src/transfers.jl:133-154``)."""

    def __init__(self, fine_space, coarse_space):
        from hfk.fespace import transfer_matrices

        self.E, self.Einj = transfer_matrices(fine_space.Q, coarse_space.Q)
        self.nf, self.nc = fine_space.nfree, coarse_space.nfree
        self.h = lib().o_transfer_create(fine_space.mesh.ncells, fine_space.nn, coarse_space.nn, _d(self.E),
                                         _d(self.Einj), _i(fine_space.cell_dof_ids), _i(coarse_space.cell_dof_ids),
                                         self.nf, self.nc)

    def __del__(self):
        if getattr(self, "h", None):
            lib().o_transfer_free(self.h)
            self.h = None

    def prolongate(self, xc):
        yf = np.zeros(self.nf)
        lib().o_prolongate(self.h, _d(np.ascontiguousarray(xc, float)), _d(yf))
        return yf

    def restrict(self, yf):
        yc = np.zeros(self.nc)
        lib().o_restrict(self.h, _d(np.ascontiguousarray(yf, float)), _d(yc))
        return yc

    def inject(self, xf, df, nfc, ndc):
        xc = np.zeros(nfc)
        dc = np.zeros(ndc)
        lib().o_inject(self.h, _d(np.ascontiguousarray(xf, float)), _d(np.ascontiguousarray(df, float)), _d(xc), _d(dc))
        return xc, dc


# ---------------------------------------------------------------------------------------------
# Solver level (src/smoothers.jl, src/preconditioners.jl:350-389, src/pmultigrid.jl, src/solvers.jl)

def chebyshev_start(n):
    """Fixed start vector sin(1 + 0.7 i) + 0.3 cos(2.3 i), normalised (``src/smoothers.jl:68-71``)."""
    i = np.arange(1, n + 1, dtype=float)
    v = np.sin(1.0 + 0.7 * i) + 0.3 * np.cos(2.3 * i)
    return v / np.linalg.norm(v)


def chebyshev_damping(degree, rng):
    """1/T_k(theta/delta) on [b/range, b] (``src/smoothers.jl:35-40``)."""
    b = 1.0
    a = b / rng
    th, de = (b + a) / 2, (b - a) / 2
    return 1.0 / np.cosh(degree * np.arccosh(th / de))


def arnoldi_bounds(apply_op, apply_prec, b, k, inner="euclidean"):
    """Ritz bounds of J P^-1 after k Arnoldi steps from b (``eigenvalue_bounds``, src/preconditioners.jl:374-389).

    Modified Gram-Schmidt Arnoldi; a (near) breakdown at step j (|H[j+1,j]| <= 1e-8 max(1, max|H[1:j,1:j]|))
    truncates the Hessenberg matrix; returns (min, max) of the real parts of its eigenvalues.
    ``inner="preconditioner"`` is the engine's option that orthogonalises in the P^-1 inner product
    <u, v> = u . P^-1 v, in which J P^-1 is self-adjoint: H is then symmetric and its Ritz values lie
    inside the spectrum (a Lanczos estimate).
    """
    n = len(b)
    k = min(k, n)
    V = np.zeros((n, k + 1))
    H = np.zeros((k + 1, k))
    if inner == "preconditioner":
        Z = np.zeros((n, k + 1))  # Z = P^-1 V
        z = apply_prec(b)
        nb = np.sqrt(max(b @ z, 0.0))
        V[:, 0], Z[:, 0] = b / nb, z / nb
        for j in range(k):
            w = apply_op(Z[:, j])
            pw = apply_prec(w)
            for i in range(j + 1):
                H[i, j] = Z[:, i] @ w
                w = w - H[i, j] * V[:, i]
                pw = pw - H[i, j] * Z[:, i]
            H[j + 1, j] = np.sqrt(max(w @ pw, 0.0))
            if H[j + 1, j] == 0:
                break
            V[:, j + 1], Z[:, j + 1] = w / H[j + 1, j], pw / H[j + 1, j]
    else:
        V[:, 0] = b / np.linalg.norm(b)
        for j in range(k):
            w = apply_op(apply_prec(V[:, j]))
            for i in range(j + 1):
                H[i, j] = V[:, i] @ w
                w = w - H[i, j] * V[:, i]
            H[j + 1, j] = np.linalg.norm(w)
            if H[j + 1, j] == 0:
                break
            V[:, j + 1] = w / H[j + 1, j]
    jj = k
    for i in range(1, k):
        if abs(H[i, i - 1]) <= 1e-8 * max(1.0, np.max(np.abs(H[:i, :i]))):
            jj = i
            break
    ev = np.linalg.eigvals(H[:jj, :jj]).real
    return ev.min(), ev.max(), H[:k + 1, :k]


class OracleChebyshev:
    """``ChebyshevState`` (src/smoothers.jl:42-146) on an oracle problem prepared at its state."""

    def __init__(self, prob: OracleProblem, degree=2, rng=20.0, inflate=1.1, eig_iters=10, eig_inner="euclidean"):
        self.prob, self.degree, self.range, self.inflate, self.eig_iters = prob, degree, rng, inflate, eig_iters
        self.eig_inner = eig_inner
        self.update()

    def update(self):
        p = self.prob
        _, _, Binv = p.blocks()
        self.blocks_ok = bool(np.all(np.isfinite(Binv)))
        if not self.blocks_ok:
            self.ok = False
            return
        lmin, lmax, _ = arnoldi_bounds(p.mf_apply, p.blocks_apply, chebyshev_start(p.nfree), self.eig_iters,
                                       self.eig_inner)
        self.lmin, self.lmax = lmin, lmax
        self.ok = bool(np.isfinite(lmax) and lmax > 0 and lmin > 0)
        self.b = self.inflate * lmax
        self.a = self.b / self.range

    def smooth(self, x, rhs, zero_guess=False, want_residual=False):
        """``smooth!`` (src/smoothers.jl:116-146); returns (x, residual or None)."""
        p = self.prob
        a, b = self.a, self.b
        th, de = (b + a) / 2, (b - a) / 2
        sg = th / de
        if zero_guess:
            x = np.zeros_like(rhs)
            r = rhs.copy()
        else:
            r = rhs - p.mf_apply(x)
        z = p.blocks_apply(r)
        rho = 1 / sg
        d = z / th
        k = self.degree
        for i in range(1, k + 1):
            x = x + d
            if i == k and not want_residual:
                break
            z = p.mf_apply(d)
            r = r - z
            if i == k:
                break
            z = p.blocks_apply(r)
            rn = 1 / (2 * sg - rho)
            d = rn * rho * d + (2 * rn / de) * z
            rho = rn
        return x, (r if want_residual else None)


class OraclePMG:
    """p-multigrid V-cycle (``PMultigrid``/``vcycle!``, src/pmultigrid.jl:256-338) on oracle levels.

    ``spaces`` finest first; ``quad`` is the working quadrature, used on every level (the coarse
    operators are captured from the Newton's forms, src/pmultigrid.jl:244-247).
    """

    def __init__(self, spaces, quad, law=LAW_SVK, params=(2.0, 1.0), degree=2, rng=20.0, inflate=1.1, eig_iters=10,
                 coarse="direct", coarse_iters=20, eig_inner="euclidean"):
        self.spaces = spaces
        self.levels = [OracleProblem(s, quad, law, params) for s in spaces]
        self.P = [OracleTransfer(spaces[l], spaces[l + 1]) for l in range(len(spaces) - 1)]
        self.cheb_cfg = (degree, rng, inflate, eig_iters, eig_inner)
        self.coarse, self.coarse_iters = coarse, coarse_iters
        self.smoothers = None
        self.xs = None

    def update(self, xf, df):
        """``update_levels!`` (src/pmultigrid.jl:168-221) + smoother updates: inject, prepare, assemble coarse."""
        xs, ds = [xf], [df]
        for l, P in enumerate(self.P):
            s = self.spaces[l + 1]
            xc, dc = P.inject(xs[-1], ds[-1], s.nfree, s.ndir)
            xs.append(xc)
            ds.append(dc)
        self.xs, self.ds = xs, ds
        for l, p in enumerate(self.levels[:-1]):
            p.mf_prepare(xs[l], ds[l])
        c = self.levels[-1]
        if self.coarse == "cg":
            # the engine's inexact coarse solve (HFK_COARSE_CG): matrix-free coarse level, blocks
            c.mf_prepare(xs[-1], ds[-1])
            _, _, Binv = c.blocks()
            self.coarse_ok = bool(np.all(np.isfinite(Binv)))
        else:
            A = c.jacobian(xs[-1], ds[-1])
            self.coarse_ok = bool(np.all(np.isfinite(A.data)))
            self.lu = spla.splu(A.tocsc()) if self.coarse_ok else None
        self.smoothers = [OracleChebyshev(p, *self.cheb_cfg) for p in self.levels[:-1]]
        self.ok = self.coarse_ok and all(s.ok for s in self.smoothers)

    def coarse_cg(self, b):
        """``coarse_iters`` block-Jacobi CG steps from zero (the engine's HFK_COARSE_CG): alpha and
        beta are 0 where their denominator is not positive."""
        c = self.levels[-1]
        x = np.zeros_like(b)
        r = b.copy()
        z = c.blocks_apply(r)
        p = z.copy()
        rz = r @ z
        for it in range(self.coarse_iters):
            q = c.mf_apply(p)
            pq = p @ q
            a = rz / pq if pq > 0 else 0.0
            x = x + a * p
            r = r - a * q
            if it + 1 == self.coarse_iters:
                break
            z = c.blocks_apply(r)
            zr = z @ r
            beta = zr / rz if rz > 0 else 0.0
            rz = zr
            p = z + beta * p
        return x

    def vcycle(self, b, level=0):
        if level == len(self.levels) - 1:
            return self.coarse_cg(b) if self.coarse == "cg" else self.lu.solve(b)
        S, P = self.smoothers[level], self.P[level]
        x, r = S.smooth(None, b, zero_guess=True, want_residual=True)
        bc = P.restrict(r)
        xc = self.vcycle(bc, level + 1)
        x = x + P.prolongate(xc)
        x, _ = S.smooth(x, b)
        return x

    def ldiv(self, r):
        if not self.ok:
            return np.full_like(r, np.nan)
        return self.vcycle(r)


def pcg(apply_op, b, prec=None, rtol=1e-8, atol=0.0, maxiter=500, x0=None):
    """Preconditioned CG with the true-residual stopping test ||b - Ax|| <= atol + rtol ||b||.

    Flexible (Polak-Ribiere) beta, so a variable preconditioner is allowed; with a fixed SPD
    preconditioner it is the CG that ``MatrixFreeSolver(krylov = :cg)`` runs (src/solvers.jl:128-148).
    Returns (x, iters, converged, relres).
    """
    x = np.zeros_like(b) if x0 is None else x0.copy()
    r = b - apply_op(x) if x0 is not None else b.copy()
    nb = np.linalg.norm(b)
    tol = atol + rtol * nb
    if np.linalg.norm(r) <= tol:
        return x, 0, True, np.linalg.norm(r) / max(nb, 1e-300)
    z = prec(r) if prec is not None else r.copy()
    p = z.copy()
    rz = r @ z
    it = 0
    while it < maxiter:
        it += 1
        Ap = apply_op(p)
        pAp = p @ Ap
        if not pAp > 0:
            return x, it, False, np.nan
        alpha = rz / pAp
        x = x + alpha * p
        rn = r - alpha * Ap
        res = np.linalg.norm(rn)
        if res <= tol:
            return x, it, True, res / nb
        zn = prec(rn) if prec is not None else rn.copy()
        rzn = rn @ zn
        beta = (zn @ (rn - r)) / rz
        p = zn + beta * p
        r, z, rz = rn, zn, rzn
    return x, it, False, np.linalg.norm(r) / nb


def gmres(apply_op, b, prec=None, rtol=1e-8, atol=0.0, maxiter=500, restart=50, flexible=True, x0=None):
    """Restarted GMRES with right preconditioning (A N^-1 u = b, x = N^-1 u), the method of
    ``MatrixFreeSolver(krylov = :gmres / :fgmres)`` (src/solvers.jl:128-131, Krylov.jl gmres!/fgmres!),
    restated after Saad's (F)GMRES: Arnoldi by classical Gram-Schmidt with one reorthogonalisation,
    Givens rotations, a cycle ends when the residual estimate meets atol + rtol ||b|| or after
    ``restart`` iterations; then x += Z y (flexible: the preconditioned basis) or x += N^-1 V y, and
    the true residual decides convergence or the next cycle. Returns (x, iters, converged, relres).
    """
    M = prec if prec is not None else (lambda v: v.copy())
    x = np.zeros_like(b) if x0 is None else x0.copy()
    nb = np.linalg.norm(b)
    tol = atol + rtol * nb
    m = min(restart, maxiter)
    r = b - apply_op(x)
    beta = np.linalg.norm(r)
    it = 0
    while beta > tol and it < maxiter:
        V = [r / beta]
        Z = []
        H = np.zeros((m + 1, m))
        cs, sn = np.zeros(m), np.zeros(m)
        g = np.zeros(m + 1)
        g[0] = beta
        jend = 0
        for j in range(m):
            if it >= maxiter:
                break
            z = M(V[j])
            Z.append(z)
            w = apply_op(z)
            Vm = np.array(V).T
            h = Vm.T @ w
            w = w - Vm @ h
            h2 = Vm.T @ w
            w = w - Vm @ h2
            h = h + h2
            hn = np.linalg.norm(w)
            col = np.zeros(m + 1)
            col[: j + 1] = h
            col[j + 1] = hn
            for i in range(j):
                t = cs[i] * col[i] + sn[i] * col[i + 1]
                col[i + 1] = -sn[i] * col[i] + cs[i] * col[i + 1]
                col[i] = t
            rr = np.hypot(col[j], col[j + 1])
            cs[j], sn[j] = (col[j] / rr, col[j + 1] / rr) if rr > 0 else (1.0, 0.0)
            col[j], col[j + 1] = rr, 0.0
            H[:, j] = col
            g[j + 1] = -sn[j] * g[j]
            g[j] = cs[j] * g[j]
            it += 1
            jend = j + 1
            if abs(g[j + 1]) <= tol or not hn > 0:
                break
            V.append(w / hn)
        y = np.zeros(jend)
        for i in range(jend - 1, -1, -1):
            y[i] = (g[i] - H[i, i + 1:jend] @ y[i + 1:]) / H[i, i] if H[i, i] != 0 else 0.0
        if flexible:
            x = x + np.array(Z[:jend]).T @ y
        else:
            x = x + M(np.array(V[:jend]).T @ y)
        r = b - apply_op(x)
        beta = np.linalg.norm(r)
    return x, it, beta <= tol, beta / max(nb, 1e-300)


# ---------------------------------------------------------------------------------------------
# MLP of the learned correction (the engine's hfk_mlp_*): numpy forward/backward with the same
# parameter layout and the BF16 rounding of the weights the GPU forward pass reads.

MLP_IN, MLP_W, MLP_OUT = 16, 64, 3


def bf16_round(w):
    """Round float32 values to bfloat16 (round to nearest even), returned as float32."""
    w = np.ascontiguousarray(w, dtype=np.float32)
    b = w.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32)


def mlp_unpack(w):
    o = 0
    W1 = w[o:o + MLP_W * MLP_IN].reshape(MLP_W, MLP_IN); o += MLP_W * MLP_IN
    b1 = w[o:o + MLP_W]; o += MLP_W
    W2 = w[o:o + MLP_W * MLP_W].reshape(MLP_W, MLP_W); o += MLP_W * MLP_W
    b2 = w[o:o + MLP_W]; o += MLP_W
    W3 = w[o:o + MLP_OUT * MLP_W].reshape(MLP_OUT, MLP_W); o += MLP_OUT * MLP_W
    b3 = w[o:o + MLP_OUT]
    return W1, b1, W2, b2, W3, b3


def mlp_forward(w, X):
    """Outputs (n x 3) for features X (n x 16), weights rounded to BF16, float64 arithmetic."""
    W1, b1, W2, b2, W3, b3 = (a.astype(np.float64) for a in mlp_unpack(bf16_round(w)))
    a1 = np.tanh(X @ W1.T + b1)
    a2 = np.tanh(a1 @ W2.T + b2)
    return a2 @ W3.T + b3


def mlp_grad(w, X, T):
    """(gradient of mean_s |out_s - t_s|^2 w.r.t. the flat weights, loss), BF16-rounded forward."""
    W1, b1, W2, b2, W3, b3 = (a.astype(np.float64) for a in mlp_unpack(bf16_round(w)))
    n = X.shape[0]
    a1 = np.tanh(X @ W1.T + b1)
    a2 = np.tanh(a1 @ W2.T + b2)
    out = a2 @ W3.T + b3
    e = out - T
    loss = float((e * e).sum() / n)
    d3 = 2 * e / n
    gW3 = d3.T @ a2
    gb3 = d3.sum(0)
    d2 = (d3 @ W3) * (1 - a2 * a2)
    gW2 = d2.T @ a1
    gb2 = d2.sum(0)
    d1 = (d2 @ W2) * (1 - a1 * a1)
    gW1 = d1.T @ X
    gb1 = d1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return g, loss


# ---------------------------------------------------------------------------------------------
# Oseen–BDF step on Taylor–Hood P2–P1 tetrahedra (oseen_oracle.cpp)


class OracleOseen:
    """The volume terms of the reference's Oseen step (test/common.jl:164-228) on a
    ``hfk.oseen.TaylorHoodSpace``, evaluated literally per (test, trial) pair."""

    def __init__(self, space, params, un, und, unm1=None, unm1d=None, quad_m=3):
        from hfk import oseen as OS  # host module (pure numpy)

        self.space = space
        pts, w = OS.tet_quadrature(quad_m)
        N2, dN2, N1, dN1, H2 = OS.tables(pts)
        self._keep = (w, N2, dN2, N1, dN1, H2)
        prm = np.ascontiguousarray(params.array())
        self.ids = space.cell_dof_ids
        self.h = lib().o_oseen_create(space.mesh.ncells, len(w), _d(w), _d(N2), _d(dN2), _d(H2), _d(N1), _d(dN1),
                                      _d(space.mesh.coords), _i(self.ids), space.nfree, space.ndir, _d(prm))
        if not self.h:
            raise RuntimeError("oracle: more than 128 colours")
        unm1 = un if unm1 is None else unm1
        unm1d = und if unm1d is None else unm1d
        self._hist = [np.ascontiguousarray(a, dtype=float) for a in (un, und, unm1, unm1d)]
        lib().o_oseen_set_history(self.h, *[_d(a) for a in self._hist])
        self.nnz = None

    def __del__(self):
        if getattr(self, "h", None):
            lib().o_oseen_free(self.h)
            self.h = None

    def set_outlet(self, facets, Pc=0.7, ZA=2.3):
        """The outlet boundary group (a ``hfk.oseen.OutletFacets``), the reference's Pc and ZA."""
        self._outlet = (facets.cells, facets.faces, np.ascontiguousarray(facets.areas), facets.normals,
                        np.ascontiguousarray(facets.w), facets.N)
        c, fa, ar, nr, w, N = self._outlet
        lib().o_oseen_set_outlet(self.h, facets.nfacets, _i(c), _i(fa), _d(ar), _d(np.asfortranarray(nr)), facets.nq,
                                 _d(w), _d(N), Pc, ZA)

    def element(self, cell):
        Ke = np.zeros((34, 34), order="F")
        Fe = np.zeros(34)
        lib().o_oseen_element(self.h, cell, _d(Ke), _d(Fe))
        return Ke, Fe

    def pattern(self):
        if self.nnz is None:
            self.nnz = int(lib().o_oseen_pattern(self.h))
            n = self.space.nfree
            self.colptr = np.zeros(n + 1, dtype=np.int64)
            self.rowval = np.zeros(self.nnz, dtype=np.int64)
            lib().o_oseen_pattern_get(self.h, _l(self.colptr), _l(self.rowval), None)
        return self.colptr, self.rowval

    def residual(self, x, dvals, nthreads=0):
        b = np.zeros(self.space.nfree)
        lib().o_oseen_residual(self.h, _d(np.ascontiguousarray(x, float)), _d(np.ascontiguousarray(dvals, float)),
                               _d(b), nthreads)
        return b

    def jacobian_values(self, nthreads=0, out=None):
        """The CSC values (zero-filled first by the restatement); ``out``: nnz float64 entries to
        assemble into in place."""
        self.pattern()
        nz = np.zeros(self.nnz) if out is None else out
        assert nz.dtype == np.float64 and nz.size == self.nnz and nz.flags.c_contiguous
        lib().o_oseen_jacobian(self.h, _d(nz), nthreads)
        return nz

    def jacobian(self, nthreads=0):
        nz = self.jacobian_values(nthreads)
        n = self.space.nfree
        return sp.csc_matrix((nz, self.rowval - 1, self.colptr - 1), shape=(n, n))
