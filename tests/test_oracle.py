"""Pins the CPU oracle with the reference's own known-answer and property tests (restated).

The reference ships no golden vectors (its tests compare against a live Gridap, which cannot run
here), so the oracle is pinned by the properties its test suite checks. Each test cites the
reference test it restates.
"""
import math

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import reldiff, svk_space, svk_state

import oracle as O
from hfk.fespace import CartesianMesh, Quadrature, VectorLagrangeSpace, gauss1d, lagrange1d, lagrange_tables, transfer_matrices


def test_lagrange1d_partition_of_unity_and_kronecker():
    # test/test_matrixfree.jl:9-17
    for Q in range(1, 5):
        for xi in (0.0, 0.3, 1.0):
            N, dN = lagrange1d(Q, xi)
            assert abs(N.sum() - 1.0) < 1e-14
            assert abs(dN.sum()) < 1e-12
    N, _ = lagrange1d(3, 0.5)
    assert np.allclose(N, [0.0, 1.0, 0.0])


def test_gauss_rule_exactness():
    for P in range(1, 7):
        x, w = gauss1d(P)
        for k in range(2 * P):
            assert abs(w @ x**k - 1.0 / (k + 1)) < 1e-14


def test_tables_partition_of_unity_and_volume():
    # test/test_tables.jl:20, :32
    for Q in (2, 3, 4, 5):
        q = Quadrature.gauss(2 * (Q - 1))
        Nt, dNt = lagrange_tables(Q, q.points())
        assert np.allclose(Nt.sum(axis=0), 1.0, atol=1e-13)
        assert np.allclose(dNt.sum(axis=0), 0.0, atol=1e-11)
        assert abs(q.w.sum() - 1.0) < 1e-14


def test_oracle_tensor_product_structure_detected():
    # test/test_matrixfree.jl:19-45 (TPTable reproduces the ND tables)
    for order in (1, 2, 3):
        V = svk_space(order=order)
        p = O.OracleProblem(V, Quadrature.gauss(2 * order))
        assert p.has_tp


def test_point_law_tangent_is_the_derivative_of_the_stress():
    # the factorised tangent equals the exact derivative (src/factorforms.jl:256-298: random-point check)
    rng = np.random.default_rng(2)
    for law in (O.LAW_SVK, O.LAW_LINEAR):
        F = np.eye(3) + 0.2 * rng.standard_normal((3, 3))
        P, T = O.point_law(law, (2.0, 1.0), F)
        eps = 1e-6
        for k in range(3):
            for L in range(3):
                dF = np.zeros((3, 3))
                dF[k, L] = eps
                Pp, _ = O.point_law(law, (2.0, 1.0), F + dF)
                Pm, _ = O.point_law(law, (2.0, 1.0), F - dF)
                fd = (Pp - Pm) / (2 * eps)
                for c in range(3):
                    for J in range(3):
                        assert abs(T[c * 3 + J, k * 3 + L] - fd[c, J]) < 1e-7
        assert np.allclose(T, T.T, atol=1e-13)


def test_svk_stress_closed_form():
    # P = F S(E) of test/common.jl:1-8 written out in numpy
    rng = np.random.default_rng(5)
    F = np.eye(3) + 0.1 * rng.standard_normal((3, 3))
    lam, mu = 2.0, 1.0
    E = 0.5 * (F.T @ F - np.eye(3))
    S = lam * np.trace(E) * np.eye(3) + 2 * mu * E
    P, _ = O.point_law(O.LAW_SVK, (lam, mu), F)
    assert np.allclose(P, F @ S, atol=1e-14)


def test_colouring_is_conflict_free_and_first_fit():
    # test/test_assembly.jl:23-38
    V = svk_space(n=(4, 3, 2), order=2)
    p = O.OracleProblem(V, Quadrature.gauss(4))
    ids = V.cell_dof_ids
    for c in range(1, p.ncolors + 1):
        cells = np.nonzero(p.colors == c)[0]
        rows = ids[:, cells]
        rows = rows[rows > 0]
        assert len(rows) == len(np.unique(rows))
    assert p.ncolors == 8  # structured Q2 hexahedra


def test_pattern_is_symmetric_with_diagonal_and_positions_consistent():
    # test/test_assembly.jl:3-21 (pattern and nzpos consistency)
    V = svk_space(order=2)
    p = O.OracleProblem(V, Quadrature.gauss(4))
    colptr, rowval = p.pattern()
    A = sp.csc_matrix((np.ones(p.nnz), rowval - 1, colptr - 1), shape=(V.nfree, V.nfree))
    assert (A != A.T).nnz == 0
    assert np.all(A.diagonal() == 1)
    ids = V.cell_dof_ids
    ndl = V.ndl
    for cell in (0, V.mesh.ncells - 1):
        for jj in range(0, ndl, 7):
            for ii in range(0, ndl, 5):
                pos = p.nzpos[ii + ndl * jj, cell]
                r, c = ids[ii, cell], ids[jj, cell]
                if r > 0 and c > 0:
                    assert rowval[pos - 1] == r and colptr[c - 1] <= pos < colptr[c]
                else:
                    assert pos == 0


def test_jacobian_matches_finite_differences_of_the_residual():
    for order, perturb in ((1, 0.0), (2, 0.0), (2, 0.2)):
        V = svk_space(order=order, perturb=perturb)
        p = O.OracleProblem(V, Quadrature.gauss(2 * order), O.LAW_SVK, (2.0, 1.0, 0.3, -0.2, 0.5))
        x = svk_state(V, amp=1e-2)
        d = V.dirichlet_values
        A = p.jacobian(x, d)
        v = np.random.default_rng(1).standard_normal(V.nfree)
        eps = 1e-6
        fd = (p.residual(x + eps * v, d) - p.residual(x - eps * v, d)) / (2 * eps)
        assert reldiff(fd, A @ v) < 1e-8


def test_point_blocks_do_not_change_the_jacobian():
    # test/test_assembly.jl:158-179 (matrix-product Jacobian for point blocks 1, 5, 8, 27, all)
    V = svk_space(order=2)
    p = O.OracleProblem(V, Quadrature.gauss(4))
    x = svk_state(V)
    d = V.dirichlet_values
    K0 = p.element_jacobian(x, d, 3, point_block=0)
    for qb in (1, 5, 8, 12, 27):
        assert reldiff(p.element_jacobian(x, d, 3, point_block=qb), K0) < 1e-14


def test_affine_field_has_exact_gradient_and_equilibrium():
    # test/test_kernels.jl:19-39: u = A x + b gives grad u = A' exactly; a uniform stress is in
    # equilibrium, so the residual vanishes at every dof whose support is interior
    A = np.array([[0.01, 0.02, 0.03], [-0.01, 0.005, 0.0], [0.002, 0.001, 0.04]])
    for order in (1, 2, 3):
        m = CartesianMesh((3, 3, 3), perturb=0.1, seed=1)
        V = VectorLagrangeSpace(m, order, "boundary", g=lambda x: x @ A.T + np.array([1.0, 2.0, 3.0]))
        p = O.OracleProblem(V, Quadrature.gauss(2 * order + 2), O.LAW_SVK, (2.0, 1.0))
        free, d = V.interpolate(lambda x: x @ A.T + np.array([1.0, 2.0, 3.0]))
        b = p.residual(free, d)
        assert np.abs(b).max() < 1e-12


def test_matrix_free_equals_assembled():
    # test/test_matrixfree.jl:74-111 (MF vs assembled at 1e-11; 1e-9 for Q3)
    for order, tol in ((1, 1e-11), (2, 1e-11), (3, 1e-9)):
        for perturb in (0.0, 0.15):
            V = svk_space(order=order, perturb=perturb)
            p = O.OracleProblem(V, Quadrature.gauss(2 * order))
            x = svk_state(V)
            d = V.dirichlet_values
            A = p.jacobian(x, d)
            p.mf_prepare(x, d)
            v = np.random.default_rng(4).standard_normal(V.nfree)
            assert reldiff(p.mf_apply(v), A @ v) < tol


def test_blocks_from_tangents_equal_assembled_diagonal_blocks():
    # test/solvers/test_chebyshev.jl:40-62
    V = svk_space(order=2)
    p = O.OracleProblem(V, Quadrature.gauss(4))
    x = svk_state(V)
    d = V.dirichlet_values
    A = p.jacobian(x, d).toarray()
    p.mf_prepare(x, d)
    dofs, B, Binv = p.blocks()
    for k in range(len(dofs)):
        ix = dofs[k] - 1
        assert np.allclose(B[k], A[np.ix_(ix, ix)], rtol=1e-12, atol=1e-14)
        assert np.allclose(Binv[k] @ B[k], np.eye(3), atol=1e-10)


def test_chebyshev_damping_closed_form():
    # test/solvers/test_chebyshev.jl:123
    assert abs(O.chebyshev_damping(3, 20.0) - 1 / math.cosh(3 * math.acosh(21 / 19))) < 1e-15


def test_chebyshev_damps_every_eigencomponent():
    # test/solvers/test_chebyshev.jl:64-98: |p_k(lambda)| <= 1/T_k(theta/delta) on [b/range, b]
    V = svk_space(n=(2, 2, 2), order=2)
    p = O.OracleProblem(V, Quadrature.gauss(4))
    x = svk_state(V)
    d = V.dirichlet_values
    A = p.jacobian(x, d).toarray()
    p.mf_prepare(x, d)
    S = O.OracleChebyshev(p, degree=3, rng=20.0)
    dofs, B, Binv = p.blocks()
    Minv = np.zeros_like(A)
    for k in range(len(dofs)):
        ix = dofs[k] - 1
        Minv[np.ix_(ix, ix)] = Binv[k]
    lam, W = np.linalg.eig(Minv @ A)
    lam = lam.real
    damp = O.chebyshev_damping(3, 20.0)
    assert S.b >= lam.max() * (1 - 1e-8)  # the inflated Ritz estimate covers the spectrum
    for i in np.nonzero(lam >= S.a)[0]:
        e = W[:, i].real
        y, _ = S.smooth(None, A @ e, zero_guess=True)  # smoothing A x = A e from 0: error e - x
        assert np.linalg.norm(e - y) <= damp * np.linalg.norm(e) * (1 + 1e-6) + 1e-12


def test_preconditioned_arnoldi_is_symmetric_and_inside_the_spectrum():
    # the engine's HFK_EIG_PRECONDITIONED option: Arnoldi in the P^-1 inner product gives a
    # symmetric (tridiagonal) H whose Ritz values lie inside the spectrum of P^-1 J
    V = svk_space(n=(2, 2, 2), order=2)
    p = O.OracleProblem(V, Quadrature.gauss(4), O.LAW_SVK, (15.0, 0.3))
    x = svk_state(V)
    d = V.dirichlet_values
    A = p.jacobian(x, d).toarray()
    p.mf_prepare(x, d)
    dofs, B, Binv = p.blocks()
    Minv = np.zeros_like(A)
    for k in range(len(dofs)):
        ix = dofs[k] - 1
        Minv[np.ix_(ix, ix)] = Binv[k]
    lam = np.sort(np.linalg.eigvals(Minv @ A).real)
    b = O.chebyshev_start(V.nfree)
    lo, hi, H = O.arnoldi_bounds(p.mf_apply, p.blocks_apply, b, 10, "preconditioner")
    Hs = H[:10, :10]
    assert np.allclose(Hs, Hs.T, atol=1e-10 * np.abs(Hs).max())
    assert np.allclose(np.triu(Hs, 2), 0, atol=1e-10 * np.abs(Hs).max())
    assert lam[0] * (1 - 1e-10) <= lo <= hi <= lam[-1] * (1 + 1e-10)
    # the Euclidean estimate of the same operator (the reference's) has nearly the same top value
    _, hi_e, _ = O.arnoldi_bounds(p.mf_apply, p.blocks_apply, b, 10)
    assert abs(hi_e - hi) < 0.05 * hi


def test_transfers_transpose_partition_of_unity_injection():
    # test/solvers/test_transfers.jl:60-122
    for qf, qc in ((2, 1), (3, 1), (3, 2), (4, 2)):
        m = CartesianMesh((2, 3, 2))
        Vf = VectorLagrangeSpace(m, qf, ("x0", "x1"))
        Vc = VectorLagrangeSpace(m, qc, ("x0", "x1"))
        T = O.OracleTransfer(Vf, Vc)
        rng = np.random.default_rng(0)
        xc = rng.standard_normal(Vc.nfree)
        yf = rng.standard_normal(Vf.nfree)
        assert abs(T.prolongate(xc) @ yf - xc @ T.restrict(yf)) < 1e-11 * np.linalg.norm(xc) * np.linalg.norm(yf)
        E, _ = transfer_matrices(qf + 1, qc + 1)
        assert np.allclose(E.sum(axis=1), 1.0)
        # nodal interpolation of the prolongation gives back the coarse field
        xf = T.prolongate(xc)
        xc2, _ = T.inject(xf, np.zeros(Vf.ndir), Vc.nfree, Vc.ndir)
        assert np.allclose(xc2, xc, atol=1e-12)


def test_coarse_operator_is_galerkin_for_linear_forms():
    # test/solvers/test_pmultigrid_levels.jl: coarse = P^T A P for linear forms (fine quadrature)
    m = CartesianMesh((2, 2, 2))
    Vf = VectorLagrangeSpace(m, 2, "boundary")
    Vc = VectorLagrangeSpace(m, 1, "boundary")
    q = Quadrature.gauss(4)
    pf = O.OracleProblem(Vf, q, O.LAW_LINEAR, (2.0, 1.0))
    pc = O.OracleProblem(Vc, q, O.LAW_LINEAR, (2.0, 1.0))
    Af = pf.jacobian(np.zeros(Vf.nfree), np.zeros(Vf.ndir)).toarray()
    Ac = pc.jacobian(np.zeros(Vc.nfree), np.zeros(Vc.ndir)).toarray()
    T = O.OracleTransfer(Vf, Vc)
    P = np.stack([T.prolongate(e) for e in np.eye(Vc.nfree)], axis=1)
    assert reldiff(P.T @ Af @ P, Ac) < 1e-12


def test_pmg_solve_matches_direct_and_is_h_independent():
    # test/solvers/test_pmultigrid.jl:37-51: same solution as LU at 1e-8, iterations <= 30, nearly h-independent
    its = []
    for n in (2, 4):
        m = CartesianMesh((n, n, n))
        g = lambda x: np.stack([0.01 * x[:, 0], -0.02 * x[:, 1] * x[:, 2], 0.005 + 0 * x[:, 0]], axis=1)
        Vs = [VectorLagrangeSpace(m, o, "boundary", g=g if o == 2 else None) for o in (2, 1)]
        q = Quadrature.gauss(4)
        mg = O.OraclePMG(Vs, q, O.LAW_LINEAR, (2.0, 1.0, 0.3, -0.2, 0.5))
        fine = mg.levels[0]
        x = np.zeros(Vs[0].nfree)
        d = Vs[0].dirichlet_values
        b = -fine.residual(x, d)
        A = fine.jacobian(x, d)
        mg.update(x, d)
        dx, it, conv, rel = O.pcg(fine.mf_apply, b, mg.ldiv, rtol=1e-10, maxiter=200)
        assert conv
        ref = sp.linalg.spsolve(A.tocsc(), b)
        assert reldiff(dx, ref) < 1e-8
        its.append(it)
    assert all(i <= 30 for i in its)
    assert its[1] <= 1.4 * its[0] + 2


def test_oracle_mlp_gradient_matches_finite_differences():
    # pins the CPU reference of the learned correction's network (its gradient checks the GPU kernels)
    rng = np.random.default_rng(0)
    w = O.bf16_round((0.1 * rng.standard_normal(5443)).astype(np.float32)).astype(np.float64)
    X = rng.standard_normal((40, 16))
    T = rng.standard_normal((40, 3))
    g, _ = O.mlp_grad(w.astype(np.float32), X, T)

    def loss(wv):
        W1, b1, W2, b2, W3, b3 = O.mlp_unpack(wv)
        a1 = np.tanh(X @ W1.T + b1)
        a2 = np.tanh(a1 @ W2.T + b2)
        return (((a2 @ W3.T + b3) - T) ** 2).sum() / len(X)

    for i in (3, 700, 1030, 2500, 5100, 5300, 5442):
        e = np.zeros_like(w)
        e[i] = 1e-6
        fd = (loss(w + e) - loss(w - e)) / 2e-6
        assert abs(g[i] - fd) <= 1e-6 * max(1.0, abs(fd))
    assert np.array_equal(O.bf16_round(np.float32([1.0, 1.00390625, -2.5])), np.float32([1.0, 1.0, -2.5]))


def test_open_face_dirichlet_counts_of_the_assembly_case():
    # Gridap's face tags fix the face interiors only: Q2 20x10x10 with x0/x1 has 41*21*21 nodes,
    # 2*19*19 fixed nodes, 52 077 free dofs (the assembly benchmark's setting)
    V = VectorLagrangeSpace(CartesianMesh((20, 10, 10)), 2, ("x0", "x1"), open_faces=True)
    assert (V.nfree, V.ndir) == (52077, 2166)
    Vc = VectorLagrangeSpace(CartesianMesh((20, 10, 10)), 2, ("x0", "x1"))
    assert Vc.ndir == 2 * 21 * 21 * 3


@pytest.mark.parametrize("law", [O.LAW_SVK, O.LAW_LINEAR])
def test_oracle_energy_derivative_is_the_residual(law):
    # the KernelFunctional restatement: d/dε E(x + ε v) = R(x)·v (no body force)
    V = svk_space(n=(2, 2, 2), order=2, perturb=0.2)
    p = O.OracleProblem(V, Quadrature.gauss(4), law, (2.0, 1.0))
    x = svk_state(V, amp=1e-2)
    d = V.dirichlet_values
    v = np.random.default_rng(4).standard_normal(V.nfree)
    # the energy is a polynomial of degree 4 in the step: the 5-point derivative is exact for it
    E = lambda t: p.functional(x + t * v, d)
    h = 1e-3
    de = (E(-2 * h) - 8 * E(-h) + 8 * E(h) - E(2 * h)) / (12 * h)
    rv = p.residual(x, d) @ v
    assert abs(de - rv) < 1e-9 * abs(rv)
    assert 0.5 < p.functional(x, d, "min_detF") < 1.5


def test_oracle_gmres_restarted_right_preconditioned():
    # the oracle's (F)GMRES restatement: a nonsymmetric system solved to the tolerance on the true
    # residual with restarts, GMRES and FGMRES alike for a fixed preconditioner, and one iteration
    # with the exact inverse as preconditioner
    import scipy.sparse as sps

    rng = np.random.default_rng(0)
    n = 200
    A = sps.random(n, n, density=0.03, random_state=1) + sps.diags(4.0 + rng.random(n))
    A = A.tocsr()
    b = rng.standard_normal(n)
    D = 1.0 / A.diagonal()
    jac = lambda v: D * v
    for flexible in (True, False):
        x, it, conv, rel = O.gmres(lambda v: A @ v, b, jac, rtol=1e-10, restart=5, flexible=flexible)
        assert conv and np.linalg.norm(b - A @ x) <= 1e-10 * np.linalg.norm(b) * (1 + 1e-9) and it > 5
    xg, itg, _, _ = O.gmres(lambda v: A @ v, b, jac, rtol=1e-10, restart=8, flexible=False)
    xf, itf, _, _ = O.gmres(lambda v: A @ v, b, jac, rtol=1e-10, restart=8, flexible=True)
    assert itg == itf and np.abs(xg - xf).max() < 1e-8 * np.abs(xf).max()
    Ainv = sps.linalg.splu(A.tocsc())
    x, it, conv, _ = O.gmres(lambda v: A @ v, b, Ainv.solve, rtol=1e-10)
    assert conv and it == 1


def test_vcycle_is_a_symmetric_positive_definite_operator():
    # test/solvers/test_pmultigrid.jl:74-84: the cycle's matrix B (columns B e_j) is symmetric and SPD
    m = CartesianMesh((2, 2, 2))
    g = lambda x: np.stack([0.01 * x[:, 0], -0.02 * x[:, 1] * x[:, 2], 0.005 + 0 * x[:, 0]], axis=1)
    Vs = [VectorLagrangeSpace(m, o, "boundary", g=g if o == 2 else None) for o in (2, 1)]
    mg = O.OraclePMG(Vs, Quadrature.gauss(4), O.LAW_LINEAR, (2.0, 1.0))
    mg.update(np.zeros(Vs[0].nfree), Vs[0].dirichlet_values)
    B = np.stack([mg.ldiv(e) for e in np.eye(Vs[0].nfree)], axis=1)
    assert np.linalg.norm(B - B.T) <= 1e-10 * np.linalg.norm(B)
    assert np.linalg.eigvalsh((B + B.T) / 2).min() > 0


@pytest.mark.parametrize("alpha,indefinite", [(0.8, True), (0.9, False)])
def test_indefinite_tangent_gives_a_negative_ritz_value(alpha, indefinite):
    # test/solvers/test_pmultigrid.jl:231-258 (there elasticity minus a mass term; here the SVK tangent
    # under the uniform compression F = alpha I, whose compressive stress makes the shear modes
    # negative at alpha = 0.8 and leaves the tangent definite at 0.9): a negative Ritz value in the
    # smoother's estimate fails the hierarchy (the cycle returns NaN), and CG without a
    # preconditioner meets the negative curvature; the definite case converges
    m = CartesianMesh((3, 3, 3))
    g = lambda x: (alpha - 1.0) * x
    Vs = [VectorLagrangeSpace(m, o, "boundary", g=g if o == 2 else None) for o in (2, 1)]
    x, _ = Vs[0].interpolate(g)
    d = Vs[0].dirichlet_values
    mg = O.OraclePMG(Vs, Quadrature.gauss(4), O.LAW_SVK, (2.0, 1.0))
    A = mg.levels[0].jacobian(x, d).toarray()
    lam = np.linalg.eigvalsh((A + A.T) / 2)
    mg.update(x, d)
    b = np.random.default_rng(0).standard_normal(Vs[0].nfree)
    _, it, conv, _ = O.pcg(mg.levels[0].mf_apply, b, None, rtol=1e-8, maxiter=500)
    if indefinite:
        assert lam.min() < 0 < lam.max()
        assert mg.smoothers[0].lmin < 0 and not mg.ok
        assert np.all(np.isnan(mg.ldiv(b)))
        assert not conv and it == 1
    else:
        assert lam.min() > 0 and mg.ok and mg.smoothers[0].lmin > 0
        assert conv


def test_nonlinear_coarse_tangent_differs_from_galerkin_by_O_h():
    # test/solvers/test_pmultigrid_levels.jl:78-95: at a smooth state the coarse SVK tangent at the
    # injected state differs from P^T A P by a first-order term in h
    g = lambda x: np.stack([0.05 * np.sin(2 * x[:, 0]), 0.03 * x[:, 1] ** 2, 0.02 * x[:, 0] * x[:, 2]], axis=1)
    errs = []
    for k in (2, 4):
        m = CartesianMesh((k, k, k))
        Vf = VectorLagrangeSpace(m, 2, "boundary", g=g)
        Vc = VectorLagrangeSpace(m, 1, "boundary")
        q = Quadrature.gauss(4)
        pf = O.OracleProblem(Vf, q, O.LAW_SVK, (2.0, 1.0))
        pc = O.OracleProblem(Vc, q, O.LAW_SVK, (2.0, 1.0))
        x, _ = Vf.interpolate(g)
        df = Vf.dirichlet_values
        T = O.OracleTransfer(Vf, Vc)
        xc, dc = T.inject(x, df, Vc.nfree, Vc.ndir)
        Af = pf.jacobian(x, df).toarray()
        Ac = pc.jacobian(xc, dc).toarray()
        P = np.stack([T.prolongate(e) for e in np.eye(Vc.nfree)], axis=1)
        gal = P.T @ Af @ P
        errs.append(np.linalg.norm(Ac - gal) / np.linalg.norm(gal))
    assert errs[0] < 0.05
    assert errs[0] / errs[1] > 1.5


def test_embeddings_are_snapped():
    # test/solvers/test_transfers.jl:135-143: entries within 1e-7 of 0 or 1 are exactly 0 or 1
    for pc, pf in ((1, 3), (2, 3), (1, 2)):
        for M in transfer_matrices(pf + 1, pc + 1):
            e = np.asarray(M).ravel()
            assert np.all((e == 0) | (e == 1) | ((np.abs(e) > 1e-7) & (np.abs(e - 1) > 1e-7)))


def test_cell_dof_matrix_layout_and_dirichlet_ids():
    # test/test_tables.jl:46-61: components of a node contiguous per cell (ldof = c*nn + n), free ids
    # 1..nfree and Dirichlet ids -1..-ndir each used, a node's three components fixed or free together
    m = CartesianMesh((3, 2, 2))
    for order in (1, 2, 3):
        V = VectorLagrangeSpace(m, order, ("x0", "y1"))
        ids = V.cell_dof_ids.astype(np.int64)
        assert ids.shape == (3 * V.nn, m.ncells)
        assert set(np.unique(ids[ids > 0]).tolist()) == set(range(1, V.nfree + 1))
        assert set(np.unique(-ids[ids < 0]).tolist()) == set(range(1, V.ndir + 1))
        assert not (ids == 0).any()
        per_comp = ids.reshape(3, V.nn, m.ncells)
        assert np.array_equal(per_comp[0] > 0, per_comp[1] > 0) and np.array_equal(per_comp[0] > 0, per_comp[2] > 0)
        free = per_comp[0] > 0  # node-major numbering: the components of a free node are consecutive ids
        assert np.all(per_comp[1][free] == per_comp[0][free] + 1) and np.all(per_comp[2][free] == per_comp[0][free] + 2)
        # the same global node carries the same ids in every cell that holds it
        gid = {}
        for c in range(m.ncells):
            for n_ in range(V.nn):
                key = int(V.cell_nodes[c, n_])
                val = tuple(per_comp[:, n_, c])
                assert gid.setdefault(key, val) == val


@pytest.mark.parametrize("qc,qf", [(1, 2), (2, 3), (1, 3)])
def test_prolongation_is_the_exact_embedding(qc, qf):
    # test/solvers/test_transfers.jl:39-50: a field of the coarse space, prolongated, is the same field
    # in the fine space (here checked against the fine nodal interpolation of a polynomial of the
    # coarse degree, without Dirichlet dofs so that every dof takes part)
    m = CartesianMesh((2, 2, 1))
    Vc = VectorLagrangeSpace(m, qc, ())
    Vf = VectorLagrangeSpace(m, qf, ())
    assert Vc.ndir == 0 and Vf.ndir == 0

    def f(x):
        X, Y, Z = x[:, 0], x[:, 1], x[:, 2]
        p = (X ** qc) * (Y ** qc) * (Z ** qc)
        return np.stack([1 + X - 2 * Y + 0.5 * p, Z * Y - 0.3 * p, 2 - X * Z + p], axis=1)

    xc, _ = Vc.interpolate(f)
    xf, _ = Vf.interpolate(f)
    T = O.OracleTransfer(Vf, Vc)
    assert reldiff(T.prolongate(xc), xf) < 1e-12


def test_chebyshev_zero_guess_residual_output_and_options():
    # test/solvers/test_chebyshev.jl:100-126: a fixed start vector makes the interval reproducible;
    # zero_guess ignores x; the residual output is b - A x; the smoother reduces the residual; the
    # damping's closed form; invalid options rejected
    from hfk import solvers as S

    V = svk_space((3, 2, 2))
    q = Quadrature.gauss(4)
    p = O.OracleProblem(V, q, O.LAW_LINEAR, (2.0, 1.0))
    p.mf_prepare(np.zeros(V.nfree), V.dirichlet_values)
    st = O.OracleChebyshev(p, degree=2)
    st2 = O.OracleChebyshev(p, degree=2)
    assert st.ok and st.lmax == st2.lmax
    rng = np.random.default_rng(5)
    b = rng.standard_normal(V.nfree)
    x1, _ = st.smooth(np.zeros(V.nfree), b)
    x2, _ = st.smooth(rng.standard_normal(V.nfree), b, zero_guess=True)
    assert reldiff(x2, x1) < 1e-13
    x3, r = st.smooth(None, b, zero_guess=True, want_residual=True)
    assert reldiff(x3, x1) < 1e-13
    assert reldiff(r, b - p.mf_apply(x3)) < 1e-12
    assert np.linalg.norm(r) < np.linalg.norm(b)
    assert abs(S.chebyshev_damping(S.Chebyshev(degree=3, range=20.0)) - 1 / math.cosh(3 * math.acosh(21 / 19))) < 1e-15
    for bad in (dict(degree=0), dict(range=1.0), dict(inflate=0.9), dict(eig_iters=1)):
        with pytest.raises(ValueError, match="HyperFEMKernels"):
            S.Chebyshev(**bad)


def test_arnoldi_bounds_against_the_dense_spectrum():
    # test/solvers/test_matrixfree_solver.jl:172-197 (vector elasticity on Q2 in place of the 2D
    # Poisson problem): the block-Jacobi preconditioned estimate within 10 % of the dense largest
    # eigenvalue and positive smallest; without a preconditioner the operator's own spectrum; the
    # same start vector gives the same bounds; an exact preconditioner breaks down at (1, 1)
    V = svk_space((3, 2, 2))
    p = O.OracleProblem(V, Quadrature.gauss(4), O.LAW_LINEAR, (2.0, 1.0))
    x, d = np.zeros(V.nfree), V.dirichlet_values
    p.mf_prepare(x, d)
    p.blocks()
    A = p.jacobian(x, d)
    Ad = A.toarray()
    n = V.nfree
    Minv = np.stack([p.blocks_apply(e) for e in np.eye(n)], axis=1)
    lam = np.linalg.eigvals(Ad @ Minv).real
    b = O.chebyshev_start(n)
    lo, hi, _ = O.arnoldi_bounds(p.mf_apply, p.blocks_apply, b, min(30, n))
    assert 0.9 * lam.max() <= hi <= 1.1 * lam.max() and lo > 0
    lo0, hi0, _ = O.arnoldi_bounds(p.mf_apply, lambda v: v, b, min(30, n))
    lamA = np.linalg.eigvalsh((Ad + Ad.T) / 2).max()
    assert 0.9 * lamA <= hi0 <= 1.1 * lamA
    b0 = np.random.default_rng(3).standard_normal(n)
    assert O.arnoldi_bounds(p.mf_apply, p.blocks_apply, b0, 10)[:2] == O.arnoldi_bounds(p.mf_apply, p.blocks_apply, b0, 10)[:2]
    lu = sp.linalg.splu(A.tocsc())
    le = O.arnoldi_bounds(p.mf_apply, lu.solve, b0, 10)[:2]
    assert abs(le[0] - 1.0) < 1e-6 and abs(le[1] - 1.0) < 1e-6
