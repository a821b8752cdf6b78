"""Batched problems (a disjoint union of independent problems in one handle).

No reference counterpart (the reference solves one problem per operator): every batched result
is checked against the same problems solved one at a time, by the oracle (residual, products,
V-cycle) and by the engine itself (Krylov iterations, Newton).
"""
import numpy as np
import pytest

from conftest import reldiff, svk_state

from hfk import batch as B
from hfk import forms
from hfk import solvers as S
from hfk.fespace import Quadrature

import oracle as O

PROBLEMS = [B.BatchProblem(2, 2.0, 1.0), B.BatchProblem(3, 12.0, 0.4), B.BatchProblem(2, 0.7, 3.5)]


def _states(union, amp=1e-3, disp=0.05, seed=0):
    return np.concatenate([svk_state(V, seed=seed + k, amp=amp, disp=disp) for k, V in enumerate(union.spaces)])


# ---- CPU ------------------------------------------------------------------------------------


def test_union_space_layout():
    (U2, U1), g = B.cube_batch(PROBLEMS)
    assert U2.nseg == 3 and U2.nfree == sum(V.nfree for V in U2.spaces)
    assert np.array_equal(U2.seg_cells, [0, 8, 8 + 27, 8 + 27 + 8])
    assert len(g) == U2.ndir and np.array_equal(g, np.concatenate([V.dirichlet_values for V in U2.spaces]))
    ids = U2.cell_dof_ids
    for k in range(U2.nseg):
        blk = ids[:, U2.seg_cells[k]:U2.seg_cells[k + 1]]
        free = blk[blk > 0] - 1
        assert free.min() >= U2.seg_dofs[k] and free.max() < U2.seg_dofs[k + 1]
        dirs = -blk[blk < 0] - 1
        assert dirs.min() >= U2.seg_dirs[k] and dirs.max() < U2.seg_dirs[k + 1]
        # the segment's block is the problem's own numbering, shifted
        own = U2.spaces[k].cell_dof_ids
        assert np.array_equal(np.where(own > 0, own + U2.seg_dofs[k], np.where(own < 0, own - U2.seg_dirs[k], 0)), blk)
    assert U1.nseg == 3 and np.array_equal(U1.seg_cells, U2.seg_cells)
    assert np.allclose(U2.params, [[q.lam, q.mu] for q in PROBLEMS])


def test_draw_batch_is_seeded_and_in_range():
    a = B.draw_batch(256, seed=4)
    b = B.draw_batch(256, seed=4)
    assert a == b and len(a) == 256
    n = np.array([q.n for q in a])
    lam = np.array([q.lam for q in a])
    mu = np.array([q.mu for q in a])
    assert n.min() >= 8 and n.max() <= 24 and len(set(n.tolist())) > 10
    assert lam.min() >= 0.5 and lam.max() <= 20 and mu.min() >= 0.2 and mu.max() <= 5


def test_oracle_coarse_cg_approaches_the_direct_coarse_solve():
    # the oracle restatement of the inexact coarse solve: many steps converge to the LU solve
    from conftest import svk_space

    Vs = [svk_space((2, 2, 2), o) for o in (2, 1)]
    q = Quadrature.gauss(4)
    x = svk_state(Vs[0])
    direct = O.OraclePMG(Vs, q)
    direct.update(x, Vs[0].dirichlet_values)
    it = O.OraclePMG(Vs, q, coarse="cg", coarse_iters=200)
    it.update(x, Vs[0].dirichlet_values)
    bc = np.random.default_rng(1).standard_normal(Vs[1].nfree)
    assert reldiff(it.coarse_cg(bc), direct.lu.solve(bc)) < 1e-10
    few = O.OraclePMG(Vs, q, coarse="cg", coarse_iters=3)
    few.update(x, Vs[0].dirichlet_values)
    assert reldiff(few.coarse_cg(bc), direct.lu.solve(bc)) > 1e-6


# ---- GPU ------------------------------------------------------------------------------------


def _union_operator(precision="fp64"):
    from hfk.operator import KernelOperator

    (U2, U1), g = B.cube_batch(PROBLEMS)
    res, jac = forms.svk_residual(2.0, 1.0, 4), forms.svk_jacobian(2.0, 1.0, 4)
    op = KernelOperator(res, jac, U2, jacobian="matrixfree")
    return op, (U2, U1), g


@pytest.mark.gpu
def test_batched_residual_and_products_match_each_problem():
    op, (U2, _), _ = _union_operator()
    assert op.problem.nseg == 3
    x = _states(U2)
    d = U2.dirichlet_values
    b = op.residual(np.zeros(U2.nfree), x, d)
    mf = op.allocate_jacobian(x)
    op.jacobian(mf, x)
    v = np.random.default_rng(5).standard_normal(U2.nfree)
    y = mf.mul(np.zeros(U2.nfree), v)
    q = Quadrature.gauss(4)
    for k, V in enumerate(U2.spaces):
        orc = O.OracleProblem(V, q, O.LAW_SVK, (PROBLEMS[k].lam, PROBLEMS[k].mu))
        xs, ds = U2.split(x)[k], U2.split_dirichlet(d)[k]
        assert reldiff(U2.split(b)[k], orc.residual(xs, ds)) < 1e-12
        orc.mf_prepare(xs, ds)
        assert reldiff(U2.split(y)[k], orc.mf_apply(U2.split(v)[k])) < 1e-12


@pytest.mark.gpu
def test_segment_dots_and_scale():
    import torch

    op, (U2, _), _ = _union_operator()
    a = np.random.default_rng(0).standard_normal(U2.nfree)
    nrm = B.segment_norms(op.problem, a)
    ref = np.array([np.linalg.norm(s) for s in U2.split(a)])
    assert np.allclose(nrm, ref, rtol=1e-13)
    t = torch.as_tensor(a, device="cuda")
    B.segment_scale(op.problem, t, [2.0, 0.0, -1.0])
    out = t.cpu().numpy()
    for k, f in enumerate([2.0, 0.0, -1.0]):
        assert np.array_equal(U2.split(out)[k], f * U2.split(a)[k])


@pytest.mark.gpu
def test_segments_are_validated():
    import ctypes

    from hfk._lib import HFKError, call, ptr

    op, (U2, _), _ = _union_operator()
    h = op.problem.h
    bad = U2.seg_dofs.copy()
    bad[-1] += 1
    with pytest.raises(HFKError, match="dof offsets"):
        call("hfk_problem_set_segments", h, 3, ptr(bad, np.int64), ptr(U2.seg_cells, np.int32), None)
    # cells of the first problem assigned to the second segment: they touch another segment's dofs
    cells = U2.seg_cells.copy()
    cells[1] -= 1
    with pytest.raises(HFKError, match="independent"):
        call("hfk_problem_set_segments", h, 3, ptr(U2.seg_dofs, np.int64), ptr(cells, np.int32), None)
    n = ctypes.c_int()
    call("hfk_problem_segments", h, ctypes.byref(n))
    assert n.value == 3  # a rejected call leaves the segments as they were


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_batched_vcycle_matches_each_problem_with_the_oracle(precision):
    op, (U2, U1), _ = _union_operator()
    x = _states(U2)
    mf = op.allocate_jacobian(x)
    op.jacobian(mf, x)
    st = S.PMultigridState(S.PMultigrid([U2, U1], S.Chebyshev(degree=3), precision=precision, coarse="cg",
                                        coarse_iters=12), mf)
    assert st.ok
    r = np.random.default_rng(2).standard_normal(U2.nfree)
    y = st.ldiv(np.zeros(U2.nfree), r)
    y2 = st.ldiv(np.zeros(U2.nfree), r)  # replayed from the captured graph (atomic scatter: last bits vary)
    assert reldiff(y2, y) < (1e-12 if precision == "fp64" else 1e-5)
    q = Quadrature.gauss(4)
    tol = 1e-9 if precision == "fp64" else 1e-4
    for k in range(U2.nseg):
        mg = O.OraclePMG([U2.spaces[k], U1.spaces[k]], q, O.LAW_SVK, (PROBLEMS[k].lam, PROBLEMS[k].mu), degree=3,
                         coarse="cg", coarse_iters=12)
        mg.update(U2.split(x)[k], U2.split_dirichlet(U2.dirichlet_values)[k])
        assert reldiff(U2.split(y)[k], mg.ldiv(U2.split(r)[k])) < tol, k


@pytest.mark.gpu
def test_batched_solve_matches_each_problem_solved_alone():
    from hfk.operator import KernelOperator

    op, (U2, U1), _ = _union_operator()
    x = _states(U2)
    mf = op.allocate_jacobian(x)
    op.jacobian(mf, x)
    b = -op.residual(np.zeros(U2.nfree), x)
    pm = dict(smoother=S.Chebyshev(degree=3), coarse="cg", coarse_iters=12)
    ls = S.MatrixFreeSolver(krylov="fcg", rtol=1e-10, preconditioner=S.PMultigrid([U2, U1], **pm))
    ns = S.numerical_setup(ls, mf)
    v = np.random.default_rng(7).standard_normal(U2.nfree)
    y_before = mf.mul(np.zeros(U2.nfree), v)
    dx = S.solve(np.zeros(U2.nfree), ns, b)
    res = ns.batched
    assert res.converged.all() and S.linear_converged(ns)
    assert res.sweeps == res.iters.max()
    assert len(set(res.iters.tolist())) > 1  # problems converge at different sweeps (skipped once done)
    # the skip flags are all reset after the solve: the product covers every problem again
    assert reldiff(mf.mul(np.zeros(U2.nfree), v), y_before) < 1e-14
    for k in range(U2.nseg):
        V2, V1 = U2.spaces[k], U1.spaces[k]
        f = (forms.svk_residual(PROBLEMS[k].lam, PROBLEMS[k].mu, 4), forms.svk_jacobian(PROBLEMS[k].lam, PROBLEMS[k].mu, 4))
        opk = KernelOperator(*f, V2, jacobian="matrixfree")
        xk = U2.split(x)[k]
        mfk = opk.allocate_jacobian(xk)
        opk.jacobian(mfk, xk)
        lsk = S.MatrixFreeSolver(krylov="fcg", rtol=1e-10, preconditioner=S.PMultigrid([V2, V1], **pm))
        nsk = S.numerical_setup(lsk, mfk)
        dk = S.solve(np.zeros(V2.nfree), nsk, U2.split(b)[k])
        assert abs(S.linear_iterations(nsk) - res.iters[k]) <= 1, (k, S.linear_iterations(nsk), res.iters)
        assert reldiff(U2.split(dx)[k], dk) < 1e-8
        assert res.relres[k] <= 1e-10 * 1.01


@pytest.mark.gpu
def test_device_driven_batched_loop_equals_the_host_loop():
    # the iterations after the second as one CUDA graph launch looping on the device (default)
    # against the host-driven loop: the same iterates, counts and residuals
    op, (U2, U1), _ = _union_operator()
    x = _states(U2)
    mf = op.allocate_jacobian(x)
    op.jacobian(mf, x)
    b = -op.residual(np.zeros(U2.nfree), x)
    pm = dict(smoother=S.Chebyshev(degree=3), coarse="cg", coarse_iters=12)
    out = {}
    for graph in (False, True):
        op.problem.set_solve_graph(graph)
        ls = S.MatrixFreeSolver(krylov="fcg", rtol=1e-10, preconditioner=S.PMultigrid([U2, U1], **pm))
        ns = S.numerical_setup(ls, mf)
        dx = S.solve(np.zeros(U2.nfree), ns, b)
        res = ns.batched
        assert res.converged.all() and res.sweeps > 2
        out[graph] = (dx, res.iters.copy(), res.sweeps, res.relres.copy())
    op.problem.set_solve_graph(True)
    assert np.array_equal(out[True][1], out[False][1]) and out[True][2] == out[False][2]
    assert reldiff(out[True][0], out[False][0]) < 1e-14
    # the true residuals (about 4e-11 of b: round-off after cancellation, with the atomic scatter's
    # add order free from run to run) agree to a few digits and meet the tolerance either way
    assert np.allclose(out[True][3], out[False][3], rtol=1e-4, atol=0)
    assert (out[True][3] <= 1e-10 * 1.01).all()
    # a limit reached inside the device loop stops it there
    op.problem.set_solve_graph(True)
    ls = S.MatrixFreeSolver(krylov="fcg", rtol=1e-14, maxiter=5, preconditioner=S.PMultigrid([U2, U1], **pm))
    ns = S.numerical_setup(ls, mf)
    S.solve(np.zeros(U2.nfree), ns, b)
    assert ns.batched.sweeps == 5 and not ns.batched.converged.any()


@pytest.mark.gpu
def test_batched_newton_matches_each_problem_solved_alone():
    from hfk.newton import newton_solve
    from hfk.operator import KernelOperator

    op, (U2, U1), g = _union_operator()
    pm = dict(smoother=S.Chebyshev(degree=3), coarse="cg", coarse_iters=12)
    ls = S.MatrixFreeSolver(krylov="fcg", rtol=1e-9, preconditioner=S.PMultigrid([U2, U1], **pm))
    loads = [0.5, 1.0]
    x, st = B.newton_solve_batched(op, ls, g, loads, rtol_newton=1e-9)
    assert st.converged.all() and (st.newton_iters >= 2).all()
    xs = x.cpu().numpy()
    for k in range(U2.nseg):
        V2, V1 = U2.spaces[k], U1.spaces[k]
        f = (forms.svk_residual(PROBLEMS[k].lam, PROBLEMS[k].mu, 4), forms.svk_jacobian(PROBLEMS[k].lam, PROBLEMS[k].mu, 4))
        opk = KernelOperator(*f, V2, jacobian="matrixfree")
        lsk = S.MatrixFreeSolver(krylov="fcg", rtol=1e-9, preconditioner=S.PMultigrid([V2, V1], **pm))
        xk, stk = newton_solve(opk, lsk, V2.dirichlet_values.copy(), loads, rtol_newton=1e-9)
        assert stk.converged and stk.newton_iters == st.newton_iters[k]
        assert reldiff(U2.split(xs)[k], xk.cpu().numpy()) < 1e-9


@pytest.mark.gpu
def test_learned_correction_is_accepted_per_problem():
    from hfk import learned

    op, (U2, U1), _ = _union_operator()
    x = _states(U2)
    mf = op.allocate_jacobian(x)
    op.jacobian(mf, x)
    st = S.PMultigridState(S.PMultigrid([U2, U1], S.Chebyshev(degree=3), coarse="cg", coarse_iters=8), mf)
    import torch

    rhs = torch.as_tensor(np.random.default_rng(3).standard_normal(U2.nfree), device="cuda")
    feats, targets = learned.collect_samples(st, mf, rhs, cycles=2)
    nb = U2.nfree // 3  # one block per node with free dofs (x0/x1 fix whole nodes)
    assert feats.shape[0] == 2 * nb
    assert torch.isfinite(feats).all() and torch.isfinite(targets).all()
    # log lambda, log mu features are per problem (blocks are numbered problem after problem)
    counts = [V.nfree // 3 for V in U2.spaces]
    f = feats[:nb].cpu().numpy()
    assert np.allclose(np.exp(f[:, 12]), np.repeat([q.lam for q in PROBLEMS], counts), rtol=1e-6)
    assert np.allclose(np.exp(f[:, 13]), np.repeat([q.mu for q in PROBLEMS], counts), rtol=1e-6)
    net = learned.MLP(seed=1)
    net.train(feats, targets, steps=50, batch=512, lr=2e-3)
    learned.attach(st, net)
    r = np.random.default_rng(4).standard_normal(U2.nfree)
    y = st.ldiv(np.zeros(U2.nfree), r)
    s = learned.stats(st)
    assert s["tried"] == U2.nseg and 0 <= s["accepted"] <= U2.nseg
    # never worse than the plain cycle in energy (y.Ay/2 - r.y, the A-norm error up to a constant),
    # problem by problem
    learned.attach(st, None)
    y0 = st.ldiv(np.zeros(U2.nfree), r)
    Ay, Ay0 = mf.mul(np.zeros(U2.nfree), y), mf.mul(np.zeros(U2.nfree), y0)
    for k in range(U2.nseg):
        sp = lambda v: U2.split(v)[k]
        e1 = 0.5 * sp(y) @ sp(Ay) - sp(r) @ sp(y)
        e0 = 0.5 * sp(y0) @ sp(Ay0) - sp(r) @ sp(y0)
        assert e1 <= e0 + 1e-12 * abs(e0)
