"""Oseen–BDF step on Taylor–Hood P2–P1 tetrahedra (the reference's test/common.jl:164-228 volume terms).

CPU: the mesh, numbering and quadrature; the oracle's element matrix against an independent numpy
restatement of the weak form; residual/Jacobian consistency. GPU: residual and CSC Jacobian against
the oracle, pattern bit-exact.
"""
import numpy as np
import pytest

from conftest import reldiff

from hfk import oseen as OS

import oracle as O


def _case(n=2, seed=3):
    m = OS.TetMesh(n)
    V = OS.TaylorHoodSpace(m)
    un, und = V.interpolate_velocity(OS.fourier_field(seed))
    unm1, unm1d = V.interpolate_velocity(OS.fourier_field(seed + 1, amplitude=0.7))
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(V.nfree)
    return m, V, (un, und, unm1, unm1d), x


def test_mesh_numbering_and_quadrature():
    m = OS.TetMesh(32)
    V = OS.TaylorHoodSpace(m)
    assert m.ncells == 6 * 32**3
    assert V.ndof_total == 65**3 * 3 + 33**3 == 859812  # the configuration's dof count
    pts, w = OS.tet_quadrature(3)
    from math import factorial

    for a in range(6):
        for b in range(6 - a):
            for c in range(6 - a - b):
                exact = factorial(a) * factorial(b) * factorial(c) / factorial(a + b + c + 3)
                assert abs((w * pts[:, 0] ** a * pts[:, 1] ** b * pts[:, 2] ** c).sum() - exact) < 1e-15
    # every cell's free ids are valid, pressure ids after the velocity block
    ids = V.cell_dof_ids
    assert ids.max() == V.nfree and -ids.min() <= V.ndir
    assert (ids[30:] > V.nfree_u).all()
    # P2 basis: Kronecker at the nodes, partition of unity of values and gradients
    nodes = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float)
    allnodes = np.vstack([nodes, [(nodes[i] + nodes[j]) / 2 for i, j in OS.EDGES]])
    for k, xi in enumerate(allnodes):
        N, dN = OS.p2_basis(xi)
        assert np.allclose(N, np.eye(10)[k]) and np.allclose(dN.sum(axis=0), 0)


def _numpy_element(V, params, hist, cell, quad_m=3):
    """The weak form a, l of test/common.jl:200-216 for one cell, vectorised over basis pairs."""
    un, und, unm1, unm1d = hist
    pts, wq = OS.tet_quadrature(quad_m)
    X = V.mesh.coords[:, :, cell]  # (3, 4)
    J = X[:, 1:] - X[:, :1]
    iJ = np.linalg.inv(J)
    det = abs(np.linalg.det(J))
    h = (6 * np.sqrt(2) * det / 6) ** (1 / 3)
    ids = V.cell_dof_ids[:, cell]
    loc = lambda f, d: np.where(ids > 0, f[np.maximum(ids, 1) - 1], np.where(ids < 0, d[np.maximum(-ids, 1) - 1], 0.0))
    un_l, um_l = loc(un, und)[:30].reshape(3, 10), loc(unm1, unm1d)[:30].reshape(3, 10)
    rho, mu, dt = params.rho, params.mu, params.dt
    c0, c1, c2 = (1.5 / dt, 2 / dt, 0.5 / dt) if params.bdf2 else (1 / dt, 1 / dt, 0.0)
    Hs = OS.p2_hessians()
    lap = np.einsum("aKL,Kc,Lc->a", Hs, iJ, iJ)
    lapn = un_l @ lap
    K = np.zeros((34, 34))
    F = np.zeros(34)
    for q, xi in enumerate(pts):
        N2, dN2 = OS.p2_basis(xi)
        N1, dN1 = OS.p1_basis(xi)
        g2, g1 = dN2 @ iJ, dN1 @ iJ
        unq, umq = un_l @ N2, um_l @ N2
        w = 2 * unq - umq if params.bdf2 else unq
        f = c1 * unq - c2 * umq
        nrm = np.linalg.norm(unq)
        taus = ((2 * nrm / h) ** 2 + 9 * (4 * mu / (rho * h * h)) ** 2) ** -0.5
        taup, taul = taus / rho, rho * nrm * h * 0.5
        U = np.zeros((34, 3))
        G = np.zeros((34, 3, 3))  # G[k, i, j] = d u_j / d x_i
        P = np.zeros(34)
        gP = np.zeros((34, 3))
        for c in range(3):
            U[c * 10:(c + 1) * 10, c] = N2
            G[c * 10:(c + 1) * 10, :, c] = g2
        P[30:] = N1
        gP[30:] = g1
        conv = np.einsum("kji,j->ki", G, w)
        E = 0.5 * (G + G.transpose(0, 2, 1))
        div = np.einsum("kii->k", G)
        Ru = rho * c0 * U + rho * conv
        rk = rho * f + mu * lapn
        a = (rho * c0 * U @ U.T + 2 * mu * np.einsum("aij,bij->ab", E, E) + rho * U @ conv.T
             - np.outer(div, P) - np.outer(P, div) + taus * conv @ Ru.T + taus * conv @ gP.T - taup * gP @ Ru.T
             - taup * gP @ gP.T + taul * np.outer(div, div))
        dV = wq[q] * det
        K += dV * a
        F += dV * (rho * U @ f + taus * conv @ rk - taup * gP @ rk)
    return K, F


@pytest.mark.parametrize("bdf2", [True, False])
def test_oracle_element_matches_numpy_weak_form(bdf2):
    m, V, hist, _ = _case(1)
    params = OS.OseenParams(mu=0.05, dt=0.01, bdf2=bdf2)  # the reference test's ρ, μ, Δt
    orc = O.OracleOseen(V, params, *hist)
    for cell in (0, 3, 5):
        Ke, Fe = orc.element(cell)
        Kn, Fn = _numpy_element(V, params, hist, cell)
        assert reldiff(Ke, Kn) < 1e-13 and reldiff(Fe, Fn) < 1e-13


def test_oracle_residual_is_affine_with_the_jacobian():
    m, V, hist, x = _case(2)
    orc = O.OracleOseen(V, OS.OseenParams(), *hist)
    A = orc.jacobian()
    d = V.dirichlet_values
    r0 = orc.residual(np.zeros(V.nfree), d)
    r1 = orc.residual(x, d)
    assert reldiff(r1 - r0, A @ x) < 1e-12
    # without advection or history (uⁿ = 0), the velocity block is symmetric (mass + viscous)
    z = (np.zeros(V.nfree), np.zeros(V.ndir), np.zeros(V.nfree), np.zeros(V.ndir))
    A0 = O.OracleOseen(V, OS.OseenParams(), *z).jacobian().toarray()[: V.nfree_u, : V.nfree_u]
    assert np.abs(A0 - A0.T).max() < 1e-12 * np.abs(A0).max()


def test_oracle_outlet_group_is_symmetric_and_affine():
    # the outlet terms (test/common.jl:194-210): backflow and Robin parts are symmetric in (u, v);
    # the Windkessel term is a load, so r(x) - r(0) = J x still holds with the group added
    m, V, hist, x = _case(2)
    params = OS.OseenParams()
    plain = O.OracleOseen(V, params, *hist)
    orc = O.OracleOseen(V, params, *hist)
    F = OS.OutletFacets(m)
    assert F.nfacets == 2 * m.n**2 and abs(F.areas.sum() - 1) < 1e-14
    orc.set_outlet(F)
    B = (orc.jacobian() - plain.jacobian()).toarray()
    assert np.abs(B).max() > 0 and np.abs(B - B.T).max() < 1e-14 * np.abs(B).max()
    d = V.dirichlet_values
    r0, r1 = orc.residual(np.zeros(V.nfree), d), orc.residual(x, d)
    assert reldiff(r1 - r0, orc.jacobian() @ x) < 1e-12
    # at w = 0 (no history) the backflow part vanishes and the group is ZA ∫ (u·n)(v·n)
    z = (np.zeros(V.nfree), np.zeros(V.ndir), np.zeros(V.nfree), np.zeros(V.ndir))
    a, b = O.OracleOseen(V, params, *z), O.OracleOseen(V, params, *z)
    b.set_outlet(F, ZA=1.0)
    Bz = (b.jacobian() - a.jacobian()).toarray()
    nx_rows = [V.gid_u[3 * g] - 1 for g in range(V.nnodes) if V.gid_u[3 * g] > 0]
    assert np.abs(np.delete(np.delete(Bz, nx_rows, 0), nx_rows, 1)).max() < 1e-15  # only u_x·v_x on x = 1


# ---- GPU ------------------------------------------------------------------------------------


@pytest.mark.gpu
@pytest.mark.parametrize("scatter", ["coloured", "atomic"])
def test_oseen_residual_and_jacobian_match_the_oracle(scatter):
    m, V, hist, x = _case(3)
    params = OS.OseenParams()
    op = OS.OseenOperator(V, params, *hist)
    op.set_scatter(scatter)
    orc = O.OracleOseen(V, params, *hist)
    A = op.sparsity_pattern()
    cp, rv = orc.pattern()
    assert np.array_equal(A.indptr, cp - 1) and np.array_equal(A.indices, rv - 1)
    assert reldiff(op.jacobian_values(np.zeros(A.nnz)), orc.jacobian_values()) < 1e-12
    d = V.dirichlet_values
    assert reldiff(op.residual(np.zeros(V.nfree), x, d), orc.residual(x, d)) < 1e-12


@pytest.mark.gpu
def test_oseen_outlet_group_matches_the_oracle():
    m, V, hist, x = _case(3)
    params = OS.OseenParams()
    F = OS.OutletFacets(m)
    op = OS.OseenOperator(V, params, *hist)
    op.set_outlet(F, Pc=0.7, ZA=2.3)
    orc = O.OracleOseen(V, params, *hist)
    orc.set_outlet(F, Pc=0.7, ZA=2.3)
    A = op.sparsity_pattern()
    assert reldiff(op.jacobian_values(np.zeros(A.nnz)), orc.jacobian_values()) < 1e-12
    d = V.dirichlet_values
    assert reldiff(op.residual(np.zeros(V.nfree), x, d), orc.residual(x, d)) < 1e-12


@pytest.mark.gpu
def test_oseen_device_vectors_and_parameters():
    import torch

    m, V, hist, x = _case(2)
    op = OS.OseenOperator(V, OS.OseenParams(bdf2=False), *hist)
    orc = O.OracleOseen(V, OS.OseenParams(bdf2=False), *hist)
    xd = torch.as_tensor(x, device="cuda")
    dd = torch.as_tensor(V.dirichlet_values, device="cuda")
    bd = torch.zeros(V.nfree, dtype=torch.float64, device="cuda")
    op.residual(bd, xd, dd)
    assert reldiff(bd.cpu().numpy(), orc.residual(x, V.dirichlet_values)) < 1e-12
