"""The assembled coarse level's direct solve: the hand-written Cholesky over the band of the matrix
(band storage) and its block triangular solves, in place of the reference's LU of the assembled
p = 1 level (src/pmultigrid.jl:97-98, :206-211; LaggedAssembled, src/preconditioners.jl:41-97).

* a coarse level of more than 40 000 free dofs (a size the earlier dense factor refused) solved
  exactly: the slot's solve leaves a relative residual below 1e-10 against the oracle's assembled
  matrix, and CG with the up-to-date factor converges in at most 2 iterations;
* tiny and wide-band levels (a full lower triangle, partial last tiles) against a dense solve;
* the failure path of the solves' bounded waits: a test knob keeps step 0 of the forward solve from
  running, so step 1 waits on a value nothing writes; the wait runs out after a short limit, the
  kernel sets its error word and returns, and the V-cycle returns an error status (numerical
  failure is a status in the reference, src/pmultigrid.jl:331-335). Nothing faults or hangs: every
  wait in the kernel is bounded and the other steps stop as soon as they see the error word.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import reldiff, svk_state

import oracle as O
from hfk import _lib, forms
from hfk import solvers as S
from hfk.fespace import CartesianMesh, Quadrature, VectorLagrangeSpace
from hfk.operator import KernelOperator, MatrixFreeJacobian

pytestmark = pytest.mark.gpu


def _q1_case(n, disp=0.01):
    m = CartesianMesh(n)
    g = [lambda x: 0 * x, lambda x: np.tile([disp, 0.0, 0.0], (len(x), 1))]
    V = VectorLagrangeSpace(m, 1, ("x0", "x1"), g=g)
    res, jac = forms.svk_residual(2.0, 1.0, 2), forms.svk_jacobian(2.0, 1.0, 2)
    op = KernelOperator(res, jac, V, jacobian="matrixfree")
    orc = O.OracleProblem(V, Quadrature.gauss(2))
    return V, op, orc


def test_band_cholesky_beyond_the_old_dense_limit():
    V, op, orc = _q1_case((24, 24, 24))
    assert V.nfree > 40000
    x = svk_state(V, amp=1e-4, disp=0.01)
    mf = MatrixFreeJacobian(op)
    op.jacobian(mf, x)
    b = -op.residual(np.zeros(V.nfree), x)
    A = orc.jacobian(x, V.dirichlet_values).tocsr()
    ls = S.MatrixFreeSolver(krylov="cg", rtol=1e-10, maxiter=50, preconditioner=S.LaggedAssembled(every=1))
    ns = S.numerical_setup(S.symbolic_setup(ls, mf), mf)
    dx = S.solve(np.zeros(V.nfree), ns, b)
    assert S.linear_converged(ns) and S.linear_iterations(ns) <= 2
    assert np.linalg.norm(A @ dx - b) <= 1e-10 * np.linalg.norm(b)
    # the slot alone (one application of the factor) is the direct solve
    st = ns.prec
    y = st.ldiv(np.zeros(V.nfree), b)
    assert np.linalg.norm(A @ y - b) <= 1e-10 * np.linalg.norm(b)


@pytest.mark.parametrize("n", [(2, 1, 1), (2, 2, 2), (3, 2, 5), (6, 5, 4)])
def test_band_cholesky_small_and_wide_band(n):
    # one to a few 64-row tiles, bands that cover the whole lower triangle, partial last tiles
    V, op, orc = _q1_case(n)
    x = svk_state(V, amp=1e-4, disp=0.01)
    mf = MatrixFreeJacobian(op)
    op.jacobian(mf, x)
    A = orc.jacobian(x, V.dirichlet_values).toarray()
    st = S.SlotState(S.LaggedAssembled(every=1), mf)
    assert st.ok
    r = np.random.default_rng(5).standard_normal(V.nfree)
    assert reldiff(st.ldiv(np.zeros(V.nfree), r), np.linalg.solve(A, r)) < 1e-11


def test_coarse_wait_runs_out_and_the_cycle_reports_it():
    m = CartesianMesh((6, 6, 6))
    g = lambda x: np.stack([0.01 * x[:, 0], 0 * x[:, 0], 0 * x[:, 0]], axis=1)
    Vs = [VectorLagrangeSpace(m, o, "boundary", g=g if o == 2 else None) for o in (2, 1)]
    assert Vs[1].nfree > 128  # at least two 128-row blocks: step 1 depends on step 0
    res, jac = forms.svk_residual(2.0, 1.0, 4), forms.svk_jacobian(2.0, 1.0, 4)
    op = KernelOperator(res, jac, Vs[0], jacobian="matrixfree")
    x = svk_state(Vs[0], amp=1e-3, disp=0.0)
    mf = op.allocate_jacobian(x)
    op.jacobian(mf, x)
    st = S.PMultigridState(S.PMultigrid(Vs, S.Chebyshev(degree=2)), mf)
    assert st.ok
    r = np.random.default_rng(6).standard_normal(Vs[0].nfree)
    y_ref = st.ldiv(np.zeros(Vs[0].nfree), r)
    # a short wait limit and the forward solve's step 0 never taken
    _lib.call("hfk_pmg_test_coarse_wait", st.h, 2000, 1)
    with pytest.raises(_lib.HFKError) as e:
        st.ldiv(np.zeros(Vs[0].nfree), r)
    assert e.value.code == 7 and "timed out" in str(e.value)  # HFK_ERR_INTERNAL
    # the knob is consumed: with the default limit back, the next cycles are the plain ones again
    _lib.call("hfk_pmg_test_coarse_wait", st.h, 0, 0)
    for _ in range(3):  # uncaptured, captured, replayed
        assert reldiff(st.ldiv(np.zeros(Vs[0].nfree), r), y_ref) < 1e-14
