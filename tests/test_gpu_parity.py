"""Parity of the CUDA engine (through the C ABI) with the CPU oracle on seeded inputs.

Tolerances: FP64 results agree with the oracle to <= 1e-12 relative (different summation order:
sum factorisation vs dense tables, GPU vs CPU reductions); integer results (colours, pattern,
positions) are bit-exact. FP32 products are checked against the FP64 oracle at 2e-6 relative.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from conftest import reldiff, svk_space, svk_state

import oracle as O
from hfk import forms
from hfk.fespace import CartesianMesh, Quadrature, VectorLagrangeSpace
from hfk.operator import KernelOperator, MatrixFreeJacobian
from hfk import solvers as S

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def make(order=2, n=(3, 2, 2), perturb=0.0, law="svk", body=(0.0, 0.0, 0.0), faces=("x0", "x1"), jac="assembled"):
    V = svk_space(n=n, order=order, perturb=perturb, faces=faces)
    deg = 2 * order
    if law == "svk":
        res, jf = forms.svk_residual(2.0, 1.0, deg, body), forms.svk_jacobian(2.0, 1.0, deg)
        olaw = O.LAW_SVK
    else:
        res, jf = forms.linear_elastic_residual(2.0, 1.0, deg, body), forms.linear_elastic_jacobian(2.0, 1.0, deg)
        olaw = O.LAW_LINEAR
    op = KernelOperator(res, jf, V, V, jacobian=jac)
    orc = O.OracleProblem(V, Quadrature.gauss(deg), olaw, (2.0, 1.0) + tuple(body))
    return V, op, orc


CASES = [(1, 0.0), (2, 0.0), (2, 0.2), (3, 0.0), (4, 0.0)]


@pytest.mark.parametrize("order,perturb", CASES)
def test_colours_bit_exact(order, perturb):
    V, op, orc = make(order, perturb=perturb)
    assert np.array_equal(op.problem.colors(), orc.colors)


@pytest.mark.parametrize("order,perturb", [(1, 0.0), (2, 0.0), (2, 0.2)])
def test_pattern_and_positions_bit_exact(order, perturb):
    V, op, orc = make(order, perturb=perturb)
    colptr, rowval = op.pattern_julia()
    ocp, orv = orc.pattern()
    assert np.array_equal(colptr, ocp) and np.array_equal(rowval, orv)
    assert np.array_equal(op.nonzero_positions(), orc.nzpos)


@pytest.mark.parametrize("order,perturb", CASES)
@pytest.mark.parametrize("law", ["svk", "linear"])
def test_residual_parity(order, perturb, law):
    V, op, orc = make(order, perturb=perturb, law=law, body=(0.3, -0.2, 0.5))
    x = svk_state(V, amp=1e-2)
    b = op.residual(np.zeros(V.nfree), x)
    assert reldiff(b, orc.residual(x, V.dirichlet_values)) < TOL64


@pytest.mark.parametrize("order,perturb,kernel", [(1, 0.0, "fma"), (2, 0.0, "fma"), (2, 0.2, "fma"),
                                                  (2, 0.0, "tensor"), (2, 0.2, "tensor")])
@pytest.mark.parametrize("law", ["svk", "linear"])
def test_jacobian_parity(order, perturb, kernel, law):
    # Q2: the element blocks on the FP64 FMA pipe (default) and on the FP64 tensor cores
    V, op, orc = make(order, perturb=perturb, law=law)
    op.problem.set_assembly_kernel(kernel)
    x = svk_state(V, amp=1e-2)
    A = op.allocate_jacobian(x)
    op.jacobian(A, x)
    ref = orc.jacobian_values(x, V.dirichlet_values)
    assert reldiff(A.data, ref) < TOL64
    # a second assembly into the same matrix (zero-fill) gives the same values
    op.jacobian(A, x)
    assert reldiff(A.data, ref) < TOL64


@pytest.mark.parametrize("kernel", ["fma", "tensor"])
def test_jacobian_parity_q2_with_64_points(kernel):
    # Gauss degree 6 on Q2 cells: 64 points, so the FMA kernel's last chunk of points is partial
    V = svk_space(n=(3, 2, 2), order=2, perturb=0.1)
    op = KernelOperator(forms.svk_residual(2.0, 1.0, 6), forms.svk_jacobian(2.0, 1.0, 6), V)
    op.problem.set_assembly_kernel(kernel)
    orc = O.OracleProblem(V, Quadrature.gauss(6))
    x = svk_state(V, amp=1e-2)
    A = op.allocate_jacobian(x)
    op.jacobian(A, x)
    assert reldiff(A.data, orc.jacobian_values(x, V.dirichlet_values)) < TOL64


@pytest.mark.parametrize("order,perturb", CASES)
@pytest.mark.parametrize("mode", ["recompute", "stored"])
def test_matrix_free_product_parity(order, perturb, mode):
    V, op, orc = make(order, perturb=perturb, jac="matrixfree")
    x = svk_state(V, amp=1e-2)
    mf = MatrixFreeJacobian(op, mode)
    op.jacobian(mf, x)
    orc.mf_prepare(x, V.dirichlet_values)
    dx = np.random.default_rng(1).standard_normal(V.nfree)
    y = mf.mul(np.zeros(V.nfree), dx)
    assert reldiff(y, orc.mf_apply(dx)) < TOL64


@pytest.mark.parametrize("n,perturb,law", [((3, 2, 2), 0.0, "svk"), ((7, 5, 6), 0.25, "svk"), ((7, 5, 6), 0.0, "linear"),
                                             ((2, 1, 1), 0.0, "svk")])
@pytest.mark.parametrize("scatter", ["coloured", "atomic"])
def test_q1_warp_synchronous_product_parity(n, perturb, law, scatter):
    # the Q1 kernel (8 lanes per cell, one per Gauss point, the nodal sums by shuffles) against the
    # oracle, FP64 and FP32: affine and perturbed (trilinear) cells, a partial last warp and CTA,
    # two cells
    V = svk_space(n=n, order=1, perturb=perturb)
    if law == "svk":
        res, jf, olaw = forms.svk_residual(2.0, 1.0, 2), forms.svk_jacobian(2.0, 1.0, 2), O.LAW_SVK
    else:
        res, jf = forms.linear_elastic_residual(2.0, 1.0, 2), forms.linear_elastic_jacobian(2.0, 1.0, 2)
        olaw = O.LAW_LINEAR
    op = KernelOperator(res, jf, V, V, jacobian="matrixfree")
    orc = O.OracleProblem(V, Quadrature.gauss(2), olaw, (2.0, 1.0))
    op.problem.set_scatter(scatter)
    op.problem.set_launch("q1")
    x = svk_state(V, amp=1e-2)
    mf = MatrixFreeJacobian(op)
    op.jacobian(mf, x)
    orc.mf_prepare(x, V.dirichlet_values)
    dx = np.random.default_rng(1).standard_normal(V.nfree)
    ref = orc.mf_apply(dx)
    assert reldiff(mf.mul(np.zeros(V.nfree), dx), ref) < TOL64
    y32 = mf.mul_f32(np.zeros(V.nfree, dtype=np.float32), dx.astype(np.float32))
    assert reldiff(y32.astype(np.float64), ref) < 2e-6


def test_q1_kernel_is_an_autotuner_candidate():
    V = svk_space(n=(8, 8, 8), order=1)
    op = KernelOperator(forms.svk_residual(2.0, 1.0, 2), forms.svk_jacobian(2.0, 1.0, 2), V, V, jacobian="matrixfree")
    x = svk_state(V, amp=1e-2)
    mf = MatrixFreeJacobian(op)
    op.jacobian(mf, x)
    dx = np.random.default_rng(3).standard_normal(V.nfree)
    y = mf.mul(np.zeros(V.nfree), dx)
    assert op.problem.tuning("jv", "fp64")["kernel"] in ("line", "point", "q1")
    orc = O.OracleProblem(V, Quadrature.gauss(2))
    orc.mf_prepare(x, V.dirichlet_values)
    assert reldiff(y, orc.mf_apply(dx)) < TOL64
    with pytest.raises(Exception):  # Q2 cells: not served by the Q1 kernel
        make(2)[1].problem.set_launch("q1")


@pytest.mark.parametrize("order,perturb", CASES)
@pytest.mark.parametrize("scatter,warps", [("coloured", 8), ("atomic", 8), ("atomic", 0)])
def test_point_parallel_product_parity(order, perturb, scatter, warps):
    # the point-parallel kernel (one thread per quadrature point; one cell per CTA, or 8 warps per
    # CTA) against the oracle, FP64 and FP32, affine and perturbed (trilinear) cells, several CTAs
    # and a partial one
    V, op, orc = make(order, perturb=perturb, jac="matrixfree")
    op.problem.set_scatter(scatter)
    op.problem.set_launch("point", warps)
    x = svk_state(V, amp=1e-2)
    mf = MatrixFreeJacobian(op)
    op.jacobian(mf, x)
    orc.mf_prepare(x, V.dirichlet_values)
    dx = np.random.default_rng(1).standard_normal(V.nfree)
    ref = orc.mf_apply(dx)
    assert reldiff(mf.mul(np.zeros(V.nfree), dx), ref) < TOL64
    y32 = mf.mul_f32(np.zeros(V.nfree, dtype=np.float32), dx.astype(np.float32))
    assert reldiff(y32.astype(np.float64), ref) < 2e-6


def test_many_vectors_match_single_products():
    # hfk_mf_apply_many over pageable host, page-locked host and device vectors (the staging slots
    # are reused from the third vector on) against one hfk_mf_apply per vector
    import torch

    V, op, orc = make(2, n=(4, 3, 3), jac="matrixfree")
    op.problem.set_scatter("coloured")  # the same summation order in both paths
    x = svk_state(V, amp=1e-2)
    mf = MatrixFreeJacobian(op)
    op.jacobian(mf, x)
    rng = np.random.default_rng(7)
    dxs = [rng.standard_normal(V.nfree) for _ in range(5)]
    ins = [dxs[0], torch.from_numpy(dxs[1]).pin_memory(), torch.from_numpy(dxs[2]).cuda(),
           torch.from_numpy(dxs[3]).pin_memory(), dxs[4]]
    outs = [np.zeros(V.nfree), torch.zeros(V.nfree, dtype=torch.float64).pin_memory(),
            torch.zeros(V.nfree, dtype=torch.float64, device="cuda"), np.zeros(V.nfree),
            torch.zeros(V.nfree, dtype=torch.float64).pin_memory()]
    mf.mul_many(outs, ins)
    for d, y in zip(dxs, outs):
        y = y.cpu().numpy() if hasattr(y, "cpu") else y
        assert np.array_equal(y, mf.mul(np.zeros(V.nfree), d))
    mf.mul_many([], [])


@pytest.mark.parametrize("order", [2, 4])
def test_matrix_free_fp32_error_bounded(order):
    V, op, orc = make(order, jac="matrixfree")
    x = svk_state(V, amp=1e-2)
    mf = MatrixFreeJacobian(op)
    op.jacobian(mf, x)
    orc.mf_prepare(x, V.dirichlet_values)
    dx = np.random.default_rng(1).standard_normal(V.nfree)
    y32 = mf.mul_f32(np.zeros(V.nfree, dtype=np.float32), dx.astype(np.float32))
    assert reldiff(y32.astype(np.float64), orc.mf_apply(dx)) < 2e-6


def test_device_pointers_and_host_pointers_agree():
    import torch

    V, op, orc = make(2, jac="matrixfree")
    op.problem.set_scatter("coloured")  # deterministic summation order: bit-identical results
    x = svk_state(V)
    b_host = op.residual(np.zeros(V.nfree), x)
    xd = torch.from_numpy(x).cuda()
    dd = torch.from_numpy(np.ascontiguousarray(V.dirichlet_values)).cuda()
    bd = torch.zeros(V.nfree, dtype=torch.float64, device="cuda")
    op.residual(bd, xd, dd)
    assert np.array_equal(bd.cpu().numpy(), b_host)


@pytest.mark.parametrize("order,perturb,law", [(2, 0.0, "svk"), (2, 0.2, "svk"), (3, 0.0, "linear"), (4, 0.0, "svk")])
def test_functionals_match_the_oracle_and_the_residual(order, perturb, law):
    # KernelFunctional (src/functionals.jl:10-27): the energy's directional derivative is the residual
    V, op, orc = make(order, perturb=perturb, law=law, jac="matrixfree")
    x = svk_state(V, amp=1e-2)
    d = V.dirichlet_values
    e = op.functional(x, d, "energy")
    assert abs(e - orc.functional(x, d, "energy")) < 1e-12 * abs(e)
    dm = op.functional(x, d, "min_detF")
    assert abs(dm - orc.functional(x, d, "min_detF")) < 1e-13
    v = np.random.default_rng(3).standard_normal(V.nfree)
    E = lambda t: op.functional(x + t * v, d)  # a polynomial of degree 4 in t: the 5-point rule is exact
    h = 1e-3
    de = (E(-2 * h) - 8 * E(-h) + 8 * E(h) - E(2 * h)) / (12 * h)
    r = op.residual(np.zeros(V.nfree), x, d)
    assert abs(de - r @ v) < 1e-9 * abs(r @ v)


def test_autotuned_launch_shape_gives_the_same_product():
    V, op, orc = make(2, jac="matrixfree")
    x = svk_state(V, amp=1e-2)
    mf = MatrixFreeJacobian(op)
    op.jacobian(mf, x)
    assert op.problem.tuning("jv") is None
    dx = np.random.default_rng(5).standard_normal(V.nfree)
    y1 = mf.mul(np.zeros(V.nfree), dx)  # first AUTO call: candidates timed, the fastest kept
    t = op.problem.tuning("jv")
    assert t is not None and (t["kernel"], t["warps"]) in {("line", 2), ("line", 4), ("point", 1), ("point", 8)}
    y2 = mf.mul(np.zeros(V.nfree), dx)
    assert reldiff(y1, y2) < 1e-14 and reldiff(y1, orc.jacobian(x, V.dirichlet_values) @ dx) < TOL64


@pytest.mark.parametrize("order", [2, 4])
def test_atomic_and_coloured_scatter_agree(order):
    V, op, orc = make(order, jac="matrixfree")
    x = svk_state(V, amp=1e-2)
    mf = MatrixFreeJacobian(op)
    op.jacobian(mf, x)
    dx = np.random.default_rng(5).standard_normal(V.nfree)
    out = {}
    for mode in ("coloured", "atomic"):
        op.problem.set_scatter(mode)
        out[mode] = (mf.mul(np.zeros(V.nfree), dx), op.residual(np.zeros(V.nfree), x))
    assert reldiff(out["atomic"][0], out["coloured"][0]) < 1e-14
    assert reldiff(out["atomic"][1], out["coloured"][1]) < 1e-13
    assert reldiff(out["coloured"][0], orc.jacobian(x, V.dirichlet_values) @ dx) < TOL64


@pytest.mark.parametrize("order,perturb", CASES)
@pytest.mark.parametrize("scatter", ["atomic", "coloured"])
def test_blocks_parity(order, perturb, scatter):
    # the nodal blocks (sum-factorised on tensor-product cells) against the oracle's dense sums,
    # affine and trilinear cells, atomic and colour-by-colour accumulation
    V, op, orc = make(order, perturb=perturb, jac="matrixfree")
    op.problem.set_scatter(scatter)
    x = svk_state(V, amp=1e-2)
    mf = MatrixFreeJacobian(op)
    op.jacobian(mf, x)
    st = S.BlockJacobiState(mf)
    assert st.ok
    orc.mf_prepare(x, V.dirichlet_values)
    od, oB, oBi = orc.blocks()
    gd, gB, gBi = st.blocks()
    assert np.array_equal(gd, od)
    assert reldiff(gB, oB) < TOL64 and reldiff(gBi, oBi) < 1e-11
    r = np.random.default_rng(3).standard_normal(V.nfree)
    assert reldiff(st.ldiv(np.zeros(V.nfree), r), orc.blocks_apply(r)) < 1e-11


def test_eigenvalue_bounds_and_chebyshev_parity():
    V, op, orc = make(2, n=(3, 3, 2), jac="matrixfree")
    x = svk_state(V, amp=1e-2)
    mf = MatrixFreeJacobian(op)
    op.jacobian(mf, x)
    st = S.BlockJacobiState(mf)
    orc.mf_prepare(x, V.dirichlet_values)
    ocheb = O.OracleChebyshev(orc, degree=3)
    lo, hi = S.eigenvalue_bounds(mf, st, 10)
    assert abs(hi - ocheb.lmax) < 1e-9 * ocheb.lmax and abs(lo - ocheb.lmin) < 1e-8 * ocheb.lmax
    rhs = np.random.default_rng(0).standard_normal(V.nfree)
    xg = np.zeros(V.nfree)
    rg = np.zeros(V.nfree)
    from hfk._lib import call, ptr

    call("hfk_chebyshev_smooth", op.problem.h, ocheb.a, ocheb.b, 3, ptr(rhs), ptr(xg), 1, ptr(rg))
    xo, ro = ocheb.smooth(None, rhs, zero_guess=True, want_residual=True)
    assert reldiff(xg, xo) < 1e-11 and reldiff(rg, ro) < 1e-10


@pytest.mark.parametrize("scatter", ["atomic", "coloured"])
@pytest.mark.parametrize("qf,qc", [(2, 1), (4, 2), (3, 2), (4, 1)])
def test_transfers_parity(qf, qc, scatter):
    # the levels are tensor-product pairs, so the sum-factorised transfer kernels run; the
    # restriction adds atomically, or colour by colour (bitwise reproducible) with the coloured scatter
    m = CartesianMesh((2, 3, 2))
    Vf = VectorLagrangeSpace(m, qf, ("x0", "x1"))
    Vc = VectorLagrangeSpace(m, qc, ("x0", "x1"))
    q = Quadrature.gauss(2 * qf)
    opf = KernelOperator(forms.svk_residual(degree=2 * qf), forms.svk_jacobian(degree=2 * qf), Vf)
    opc = KernelOperator(forms.svk_residual(degree=2 * qf), forms.svk_jacobian(degree=2 * qf), Vc)
    opf.problem.set_scatter(scatter)
    P = S.Prolongation(opc.problem, opf.problem)
    T = O.OracleTransfer(Vf, Vc)
    rng = np.random.default_rng(0)
    xc, yf = rng.standard_normal(Vc.nfree), rng.standard_normal(Vf.nfree)
    assert reldiff(P.prolongate(np.zeros(Vf.nfree), xc), T.prolongate(xc)) < 1e-14
    rc = P.restrict(np.zeros(Vc.nfree), yf)
    assert reldiff(rc, T.restrict(yf)) < 1e-14
    if scatter == "coloured":
        assert np.array_equal(P.restrict(np.zeros(Vc.nfree), yf), rc)
    df = rng.standard_normal(Vf.ndir)
    xi, di = P.inject(np.zeros(Vc.nfree), np.zeros(Vc.ndir), yf, df)
    oxi, odi = T.inject(yf, df, Vc.nfree, Vc.ndir)
    assert reldiff(xi, oxi) < 1e-14 and reldiff(di, odi) < 1e-14


def _pmg_case(n, orders, law="linear"):
    m = CartesianMesh((n, n, n))
    g = lambda x: np.stack([0.01 * x[:, 0], -0.02 * x[:, 1] * x[:, 2], 0.005 + 0 * x[:, 0]], axis=1)
    Vs = [VectorLagrangeSpace(m, o, "boundary", g=g if l == 0 else None) for l, o in enumerate(orders)]
    deg = 2 * orders[0]
    body = (0.3, -0.2, 0.5)
    if law == "linear":
        res, jac = forms.linear_elastic_residual(2.0, 1.0, deg, body), forms.linear_elastic_jacobian(2.0, 1.0, deg)
    else:
        res, jac = forms.svk_residual(2.0, 1.0, deg, body), forms.svk_jacobian(2.0, 1.0, deg)
    return Vs, res, jac


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_vcycle_parity_with_oracle(precision):
    Vs, res, jac = _pmg_case(3, (2, 1), "svk")
    op = KernelOperator(res, jac, Vs[0], jacobian="matrixfree")
    x = svk_state(Vs[0], amp=0.0, disp=0.0)
    mf = op.allocate_jacobian(x)
    op.jacobian(mf, x)
    st = S.PMultigridState(S.PMultigrid(Vs, S.Chebyshev(degree=2), precision=precision), mf)
    assert st.ok
    mg = O.OraclePMG(Vs, Quadrature.gauss(4), O.LAW_SVK, (2.0, 1.0, 0.3, -0.2, 0.5), degree=2)
    mg.update(x, Vs[0].dirichlet_values)
    info = st.level_info(0)
    assert abs(info["b"] - mg.smoothers[0].b) < 1e-9 * mg.smoothers[0].b
    r = np.random.default_rng(2).standard_normal(Vs[0].nfree)
    y = st.ldiv(np.zeros(Vs[0].nfree), r)
    tol = 1e-9 if precision == "fp64" else 1e-5
    assert reldiff(y, mg.ldiv(r)) < tol


def test_vcycle_parity_with_preconditioned_eigenvalue_estimate():
    # the P^-1 inner-product Arnoldi option of the smoothers' estimate, against the oracle
    Vs, res, jac = _pmg_case(3, (2, 1), "svk")
    op = KernelOperator(res, jac, Vs[0], jacobian="matrixfree")
    x = svk_state(Vs[0], amp=0.0, disp=0.0)
    mf = op.allocate_jacobian(x)
    op.jacobian(mf, x)
    st = S.PMultigridState(S.PMultigrid(Vs, S.Chebyshev(degree=2, eig_inner="preconditioner")), mf)
    assert st.ok
    mg = O.OraclePMG(Vs, Quadrature.gauss(4), O.LAW_SVK, (2.0, 1.0, 0.3, -0.2, 0.5), degree=2,
                     eig_inner="preconditioner")
    mg.update(x, Vs[0].dirichlet_values)
    info = st.level_info(0)
    assert abs(info["lmax"] - mg.smoothers[0].lmax) < 1e-9 * mg.smoothers[0].lmax
    assert abs(info["lmin"] - mg.smoothers[0].lmin) < 1e-8 * mg.smoothers[0].lmax
    r = np.random.default_rng(2).standard_normal(Vs[0].nfree)
    assert reldiff(st.ldiv(np.zeros(Vs[0].nfree), r), mg.ldiv(r)) < 1e-9


@pytest.mark.parametrize("cross", [3, 6])
def test_banded_coarse_factor_matches_the_oracle_vcycle(cross):
    # an elongated mesh: the coarse level's band is narrow against its size, so the Cholesky factor
    # is computed block column by block column over the band (several 256-row blocks) and the
    # cycle's triangular solves run block by block (128-row blocks; cross section 3: one band tile
    # per block, 6: two, with a partial last block in both)
    m = CartesianMesh((cross, cross, 40), domain=(0.0, 1.0, 0.0, 1.0, 0.0, 10.0))
    g = lambda x: np.stack([0.01 * x[:, 2], 0 * x[:, 0], 0 * x[:, 0]], axis=1)
    Vs = [VectorLagrangeSpace(m, o, ("z0", "z1"), g=g if o == 2 else None) for o in (2, 1)]
    res, jac = forms.svk_residual(2.0, 1.0, 4), forms.svk_jacobian(2.0, 1.0, 4)
    op = KernelOperator(res, jac, Vs[0], jacobian="matrixfree")
    x = svk_state(Vs[0], amp=1e-3, disp=0.0)
    mf = op.allocate_jacobian(x)
    op.jacobian(mf, x)
    st = S.PMultigridState(S.PMultigrid(Vs, S.Chebyshev(degree=2)), mf)
    assert st.ok and Vs[1].nfree > 3 * 256
    mg = O.OraclePMG(Vs, Quadrature.gauss(4), O.LAW_SVK, (2.0, 1.0), degree=2)
    mg.update(x, Vs[0].dirichlet_values)
    r = np.random.default_rng(4).standard_normal(Vs[0].nfree)
    assert reldiff(st.ldiv(np.zeros(Vs[0].nfree), r), mg.ldiv(r)) < 1e-9


def test_pmg_follows_the_prepared_dirichlet_values():
    # the hierarchy is built at the state the Jacobian was prepared at, not at the space's values
    Vs, res, jac = _pmg_case(3, (2, 1), "svk")
    op = KernelOperator(res, jac, Vs[0], jacobian="matrixfree")
    x = np.zeros(Vs[0].nfree)
    d = 0.1 * Vs[0].dirichlet_values
    mf = op.allocate_jacobian(x)
    mf.prepare(x, d)
    st = S.PMultigridState(S.PMultigrid(Vs, S.Chebyshev(degree=2)), mf)
    mg = O.OraclePMG(Vs, Quadrature.gauss(4), O.LAW_SVK, (2.0, 1.0, 0.3, -0.2, 0.5), degree=2)
    mg.update(x, d)
    r = np.random.default_rng(3).standard_normal(Vs[0].nfree)
    assert reldiff(st.ldiv(np.zeros(Vs[0].nfree), r), mg.ldiv(r)) < 1e-9


@pytest.mark.parametrize("orders", [(2, 1), (3, 1), (4, 2, 1)])
def test_pmg_solve_matches_direct_and_iterations_bounded(orders):
    # test/solvers/test_pmultigrid.jl:37-51
    its = []
    for n in (2, 4):
        Vs, res, jac = _pmg_case(n, orders)
        op = KernelOperator(res, jac, Vs[0], jacobian="matrixfree")
        x = np.zeros(Vs[0].nfree)
        mf = op.allocate_jacobian(x)
        op.jacobian(mf, x)
        b = -op.residual(np.zeros(Vs[0].nfree), x)
        ls = S.MatrixFreeSolver(krylov="fcg", rtol=1e-10, maxiter=200, preconditioner=S.PMultigrid(Vs))
        ns = S.numerical_setup(S.symbolic_setup(ls, mf), mf)
        dx = S.solve(np.zeros(Vs[0].nfree), ns, b)
        assert S.linear_converged(ns)
        orc = O.OracleProblem(Vs[0], Quadrature.gauss(2 * orders[0]), O.LAW_LINEAR, (2.0, 1.0, 0.3, -0.2, 0.5))
        A = orc.jacobian(x, Vs[0].dirichlet_values)
        ref = sp.linalg.spsolve(A.tocsc(), b)
        assert reldiff(dx, ref) < 1e-8
        its.append(S.linear_iterations(ns))
    assert all(i <= 30 for i in its), its
    assert its[1] <= 1.4 * its[0] + 2


def test_solver_slots_reproduce_the_direct_solve():
    # test/solvers/test_matrixfree_solver.jl:24-52: GMRES, FGMRES and CG without and with the slots
    # (LaggedAssembled, BlockJacobi) reproduce the direct solve; an up-to-date LaggedAssembled is an
    # exact preconditioner (at most 2 iterations), and each slot was built once
    V, op, orc = make(2, jac="matrixfree")
    x = svk_state(V, amp=1e-2)
    mf = MatrixFreeJacobian(op)
    op.jacobian(mf, x)
    A = orc.jacobian(x, V.dirichlet_values)
    b = -op.residual(np.zeros(V.nfree), x)
    ref = sp.linalg.spsolve(A.tocsc(), b)
    n = V.nfree
    configs = [("gmres", None), ("fgmres", None), ("gmres", S.LaggedAssembled()),
               ("gmres", S.LaggedAssembled(every=2)), ("gmres", S.BlockJacobi()), ("fgmres", S.BlockJacobi()),
               ("cg", None), ("cg", S.BlockJacobi()), ("cg", S.LaggedAssembled())]
    for kry, prec in configs:
        ls = S.MatrixFreeSolver(krylov=kry, rtol=1e-10, maxiter=4000, restart=n, preconditioner=prec)
        ns = S.numerical_setup(S.symbolic_setup(ls, mf), mf)
        dx = S.solve(np.zeros(n), ns, b)
        its = S.linear_iterations(ns)
        assert S.linear_converged(ns) and reldiff(dx, ref) < 1e-8, (kry, prec)
        assert 0 < its <= n + 1
        if isinstance(prec, S.LaggedAssembled):
            assert its <= 2
        assert S.preconditioner_builds(ns) == (0 if prec is None else 1)


def test_lagged_assembled_rebuilds_every_k_setups():
    # test/solvers/test_matrixfree_solver.jl:94-112: builds at setups 1 and 4 for every = 3; the
    # stale factor still converges to each new solution; exact where rebuilt
    V, op, orc = make(2, jac="matrixfree")
    n = V.nfree
    rng = np.random.default_rng(8)
    states = [svk_state(V, amp=1e-2) + 0.01 * rng.standard_normal(n) for _ in range(5)]
    mf = MatrixFreeJacobian(op)
    op.jacobian(mf, states[0])
    ls = S.MatrixFreeSolver(krylov="gmres", rtol=1e-10, maxiter=4000, restart=n,
                            preconditioner=S.LaggedAssembled(every=3))
    ns = S.numerical_setup(S.symbolic_setup(ls, mf), mf)
    its = []
    for k, x in enumerate(states, start=1):
        if k > 1:
            op.jacobian(mf, x)
            S.numerical_setup_update(ns, mf)
        assert S.preconditioner_builds(ns) == 1 + (k - 1) // 3
        b = op.residual(np.zeros(n), x)
        dx = S.solve(np.zeros(n), ns, b)
        A = orc.jacobian(x, V.dirichlet_values)
        assert S.linear_converged(ns) and reldiff(dx, sp.linalg.spsolve(A.tocsc(), b)) < 1e-8
        its.append(S.linear_iterations(ns))
    assert its[0] <= 2 and its[3] <= 2 and all(i > 0 for i in its)


def test_lagged_coarse_newton_matches_direct_newton():
    # test/solvers/test_pmultigrid.jl:95-115: Newton with the matrix-free p-MG GMRES, the coarse level
    # rebuilt every `coarse_every` updates, against Newton with a direct solve of the assembled
    # tangent: the same number of Newton iterations, histories within half a decade, the same
    # solution, and one coarse build per `every` Newton iterations
    import math

    Vs, res, jac = _pmg_case(3, (2, 1), law="svk")

    def newton(op, solve_lin, maxiter=12, tol=1e-10):
        x = np.zeros(Vs[0].nfree)
        b = op.residual(np.zeros(Vs[0].nfree), x)
        r0 = np.linalg.norm(b)
        hist = []
        for _ in range(maxiter):
            x = x - solve_lin(op, x, b)
            b = op.residual(np.zeros(Vs[0].nfree), x)
            hist.append(np.linalg.norm(b) / r0)
            if hist[-1] < tol:
                break
        return x, hist

    def direct(op, x, b):
        A = op.allocate_jacobian(x)
        op.jacobian(A, x)
        return sp.linalg.spsolve(A.tocsc(), b)

    x_lu, h_lu = newton(KernelOperator(res, jac, Vs[0]), direct)
    for every in (1, 3):
        op = KernelOperator(res, jac, Vs[0], jacobian="matrixfree")
        ls = S.MatrixFreeSolver(krylov="gmres", rtol=1e-11, maxiter=200,
                                preconditioner=S.PMultigrid(Vs, coarse_every=every))
        state = {}

        def mf_solve(op, x, b):
            mf = state.get("mf") or op.allocate_jacobian(x)
            op.jacobian(mf, x)
            state["mf"] = mf
            ns = state.get("ns")
            ns = S.numerical_setup(S.symbolic_setup(ls, mf), mf) if ns is None else S.numerical_setup_update(ns, mf)
            state["ns"] = ns
            dx = S.solve(np.zeros(Vs[0].nfree), ns, b)
            assert S.linear_converged(ns)
            return dx

        x_mf, h_mf = newton(op, mf_solve)
        assert len(h_mf) == len(h_lu)
        assert np.all(np.abs(np.log10(h_mf) - np.log10(h_lu)) < 0.5)
        assert reldiff(x_mf, x_lu) < 1e-8
        assert S.preconditioner_builds(state["ns"]) == math.ceil(len(h_mf) / every)


@pytest.mark.parametrize("krylov", ["gmres", "fgmres"])
def test_gmres_matches_the_oracle(krylov):
    # MatrixFreeSolver(krylov = :gmres / :fgmres) (src/solvers.jl:128-131): the engine's restarted
    # right-preconditioned GMRES against the oracle's restatement with the oracle's V-cycle: the same
    # iteration count (a small restart, so that cycles restart), the same solution, the true
    # residual at the tolerance; without a preconditioner as well
    Vs, res, jac = _pmg_case(3, (2, 1))
    op = KernelOperator(res, jac, Vs[0], jacobian="matrixfree")
    x = np.zeros(Vs[0].nfree)
    mf = op.allocate_jacobian(x)
    op.jacobian(mf, x)
    b = -op.residual(np.zeros(Vs[0].nfree), x)
    orc = O.OracleProblem(Vs[0], Quadrature.gauss(4), O.LAW_LINEAR, (2.0, 1.0, 0.3, -0.2, 0.5))
    A = orc.jacobian(x, Vs[0].dirichlet_values)
    mg = O.OraclePMG(Vs, Quadrature.gauss(4), O.LAW_LINEAR, (2.0, 1.0, 0.3, -0.2, 0.5), degree=2)
    mg.update(x, Vs[0].dirichlet_values)
    flex = krylov == "fgmres"
    for prec, restart in ((S.PMultigrid(Vs), 4), (None, 20)):
        ls = S.MatrixFreeSolver(krylov=krylov, rtol=1e-10, maxiter=400, restart=restart, preconditioner=prec)
        ns = S.numerical_setup(S.symbolic_setup(ls, mf), mf)
        dx = S.solve(np.zeros(Vs[0].nfree), ns, b)
        ox, oit, oconv, orel = O.gmres(lambda v: A @ v, b, mg.ldiv if prec is not None else None, rtol=1e-10,
                                       maxiter=400, restart=restart, flexible=flex)
        assert S.linear_converged(ns) and oconv
        assert abs(S.linear_iterations(ns) - oit) <= 1, (S.linear_iterations(ns), oit)
        assert reldiff(dx, ox) < 1e-8
        assert np.linalg.norm(b - A @ dx) <= 1e-10 * np.linalg.norm(b) * (1 + 1e-6)


def test_mixed_precision_solve_reaches_fp64_tolerance():
    Vs, res, jac = _pmg_case(4, (2, 1), "svk")
    op = KernelOperator(res, jac, Vs[0], jacobian="matrixfree")
    x = np.zeros(Vs[0].nfree)
    mf = op.allocate_jacobian(x)
    op.jacobian(mf, x)
    b = -op.residual(np.zeros(Vs[0].nfree), x)
    for prec in ("fp64", "fp32"):
        ls = S.MatrixFreeSolver(krylov="fcg", rtol=1e-8, preconditioner=S.PMultigrid(Vs, precision=prec))
        ns = S.numerical_setup(ls, mf)
        dx = S.solve(np.zeros(Vs[0].nfree), ns, b)
        assert S.linear_converged(ns)
        r = b - mf @ dx
        assert np.linalg.norm(r) <= 1e-8 * np.linalg.norm(b) * 1.01


def test_nan_state_makes_the_preconditioner_fail_as_a_status():
    # test/solvers/test_pmultigrid.jl:117-133: a NaN tangent gives ok = false, NaN from ldiv, failed solve
    Vs, res, jac = _pmg_case(2, (2, 1), "svk")
    op = KernelOperator(res, jac, Vs[0], jacobian="matrixfree")
    x = np.zeros(Vs[0].nfree)
    x[5] = np.nan
    mf = op.allocate_jacobian(x)
    op.jacobian(mf, x)
    ls = S.MatrixFreeSolver(krylov="fcg", rtol=1e-8, preconditioner=S.PMultigrid(Vs))
    ns = S.numerical_setup(ls, mf)
    assert not ns.prec.ok
    y = ns.prec.ldiv(np.zeros(Vs[0].nfree), np.ones(Vs[0].nfree))
    assert np.all(np.isnan(y))
    dx = S.solve(np.zeros(Vs[0].nfree), ns, np.ones(Vs[0].nfree))
    assert not S.linear_converged(ns) and S.linear_iterations(ns) == 0


def test_update_changes_parameters_keeps_structure():
    V, op, orc = make(2)
    x = svk_state(V, amp=1e-2)
    op2 = op.update(forms.svk_residual(4.0, 0.5, 4), forms.svk_jacobian(4.0, 0.5, 4))
    assert op2.problem is op.problem
    orc.set_params((4.0, 0.5))
    assert reldiff(op2.residual(np.zeros(V.nfree), x), orc.residual(x, V.dirichlet_values)) < TOL64


def test_single_cell_and_all_dirichlet_but_one_node():
    m = CartesianMesh((1, 1, 1))
    V = VectorLagrangeSpace(m, 2, "boundary")  # one interior node: 3 free dofs
    op = KernelOperator(forms.svk_residual(), forms.svk_jacobian(), V)
    orc = O.OracleProblem(V, Quadrature.gauss(4))
    x = np.array([0.01, -0.02, 0.03])
    assert reldiff(op.residual(np.zeros(3), x), orc.residual(x, V.dirichlet_values)) < TOL64
    A = op.allocate_jacobian(x)
    op.jacobian(A, x)
    assert reldiff(A.data, orc.jacobian_values(x, V.dirichlet_values)) < TOL64


def test_newton_pmg_load_stepping_matches_oracle_newton():
    # the canonical Newton loop (test/solvers/test_pmultigrid.jl:86-115): same trajectory as the oracle
    from hfk.newton import newton_solve

    m = CartesianMesh((3, 3, 3))
    gfun = [lambda x: 0 * x, lambda x: np.tile([0.1, 0.0, 0.0], (len(x), 1))]
    Vs = [VectorLagrangeSpace(m, o, ("x0", "x1"), g=gfun if o == 2 else None) for o in (2, 1)]
    g_full = Vs[0].dirichlet_values.copy()
    res, jac = forms.svk_residual(2.0, 1.0, 4), forms.svk_jacobian(2.0, 1.0, 4)
    op = KernelOperator(res, jac, Vs[0], jacobian="matrixfree")
    loads = [0.5, 1.0]
    for prec in ("fp64", "fp32"):
        ls = S.MatrixFreeSolver(krylov="fcg", rtol=1e-10, preconditioner=S.PMultigrid(Vs, S.Chebyshev(degree=3),
                                                                                      precision=prec))
        x, st = newton_solve(op, ls, g_full, loads, rtol_newton=1e-10)
        assert st.converged and st.newton_iters >= 2
        # oracle Newton with a direct solve of the assembled tangent
        orc = O.OracleProblem(Vs[0], Quadrature.gauss(4))
        xo = np.zeros(Vs[0].nfree)
        for lam in loads:
            d = lam * g_full
            for _ in range(20):
                r = orc.residual(xo, d)
                if np.linalg.norm(r) < 1e-13:
                    break
                xo = xo - sp.linalg.spsolve(orc.jacobian(xo, d).tocsc(), r)
        assert reldiff(x.cpu().numpy(), xo) < 1e-8


@pytest.mark.parametrize("alpha,indefinite", [(0.8, True), (0.9, False)])
def test_indefinite_tangent_is_reported_by_the_solve(alpha, indefinite):
    # test/solvers/test_pmultigrid.jl:231-258, with the SVK tangent under the uniform compression
    # F = alpha I in place of the reference's elasticity-minus-mass form (indefinite at 0.8, definite
    # at 0.9): a failed p-multigrid solve that met a negative Ritz value is reported indefinite
    # (preconditioner_indefinite), CG without a preconditioner meets the negative curvature itself
    m = CartesianMesh((3, 3, 3))
    g = lambda x: (alpha - 1.0) * x
    Vs = [VectorLagrangeSpace(m, o, "boundary", g=g if o == 2 else None) for o in (2, 1)]
    res, jac = forms.svk_residual(2.0, 1.0, 4), forms.svk_jacobian(2.0, 1.0, 4)
    op = KernelOperator(res, jac, Vs[0], jacobian="matrixfree")
    x, _ = Vs[0].interpolate(g)
    mf = op.allocate_jacobian(x)
    op.jacobian(mf, x)
    b = np.random.default_rng(0).standard_normal(Vs[0].nfree)
    for krylov in ("fcg", "gmres"):
        ls = S.MatrixFreeSolver(krylov=krylov, rtol=1e-8, preconditioner=S.PMultigrid(Vs))
        ns = S.numerical_setup(S.symbolic_setup(ls, mf), mf)
        dx = np.zeros(Vs[0].nfree)
        S.solve(dx, ns, b)
        if indefinite:
            assert not S.linear_converged(ns) and S.linear_iterations(ns) == 0 and S.linear_indefinite(ns)
            assert np.all(dx == 0)
        else:
            assert S.linear_converged(ns) and not S.linear_indefinite(ns)
    ls0 = S.MatrixFreeSolver(krylov="cg", rtol=1e-8, maxiter=500)
    ns0 = S.numerical_setup(S.symbolic_setup(ls0, mf), mf)
    dx = np.zeros(Vs[0].nfree)
    S.solve(dx, ns0, b)
    assert S.linear_converged(ns0) == (not indefinite) and S.linear_indefinite(ns0) == indefinite
    assert np.all(np.isfinite(dx))
