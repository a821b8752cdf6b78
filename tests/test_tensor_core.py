"""The FP32 matrix-free product with both sum-factorisation contractions on the tensor cores
(tcgen05.mma kind::tf32, operands split hi + lo), against the FP64 oracle's product (mul!,
src/matrixfree.jl:341-424; tp_interpolate! / tp_contract!, src/tensorproduct.jl:125-224).

Tolerance: 2e-6 relative, the FP32 products' tolerance in every other test. Cases: a mesh smaller
than one CTA's 128 cells, several CTAs with a partial last one, perturbed (non-affine) cells, the
colour-by-colour launch, the SVK and linear laws; the kernels' bounded waits never run out (the
problem's device error word stays 0). The autotuner offers the kernel for the FP32 product and keeps
it only when it agrees with the line-mapped kernel.
"""
import numpy as np
import pytest

from conftest import reldiff, svk_space, svk_state

import oracle as O
from hfk import forms
from hfk.fespace import Quadrature
from hfk.operator import KernelOperator, MatrixFreeJacobian

pytestmark = pytest.mark.gpu

TOL32 = 2e-6


def _case(n, perturb=0.0, law="svk", scatter="atomic"):
    V = svk_space(n=n, order=2, perturb=perturb)
    if law == "svk":
        res, jac, olaw = forms.svk_residual(2.0, 1.0, 4), forms.svk_jacobian(2.0, 1.0, 4), O.LAW_SVK
    else:
        res, jac = forms.linear_elastic_residual(2.0, 1.0, 4), forms.linear_elastic_jacobian(2.0, 1.0, 4)
        olaw = O.LAW_LINEAR
    op = KernelOperator(res, jac, V, jacobian="matrixfree")
    op.problem.set_scatter(scatter)
    op.problem.set_launch("tensor")
    orc = O.OracleProblem(V, Quadrature.gauss(4), olaw, (2.0, 1.0))
    return V, op, orc


@pytest.mark.parametrize("n,perturb,law,scatter", [((3, 2, 2), 0.0, "svk", "atomic"),
                                                   ((12, 12, 12), 0.0, "svk", "atomic"),
                                                   ((6, 5, 7), 0.2, "svk", "atomic"),
                                                   ((6, 5, 7), 0.0, "linear", "atomic"),
                                                   ((6, 5, 7), 0.0, "svk", "coloured")])
def test_tensor_core_product_matches_the_oracle(n, perturb, law, scatter):
    V, op, orc = _case(n, perturb, law, scatter)
    x = svk_state(V, amp=1e-2)
    mf = MatrixFreeJacobian(op)
    op.jacobian(mf, x)
    orc.mf_prepare(x, V.dirichlet_values)
    dx = np.random.default_rng(1).standard_normal(V.nfree)
    ref = orc.mf_apply(dx)
    for _ in range(2):  # the second call reuses the tables
        y32 = mf.mul_f32(np.zeros(V.nfree, dtype=np.float32), dx.astype(np.float32))
        err = reldiff(y32.astype(np.float64), ref)
        assert err < TOL32, err
    assert op.problem.device_errors() == 0
    print(f"tensor-core FP32 J*v {n}, perturb {perturb}, {law}, {scatter}: relative error {err:.2e}")


def test_autotuner_offers_the_tensor_core_product():
    V = svk_space(n=(10, 10, 10), order=2)
    op = KernelOperator(forms.svk_residual(2.0, 1.0, 4), forms.svk_jacobian(2.0, 1.0, 4), V, jacobian="matrixfree")
    x = svk_state(V, amp=1e-2)
    mf = MatrixFreeJacobian(op)
    op.jacobian(mf, x)
    dx = np.random.default_rng(2).standard_normal(V.nfree).astype(np.float32)
    y = mf.mul_f32(np.zeros(V.nfree, dtype=np.float32), dx)
    tuned = op.problem.tuning("jv", "fp32")
    assert tuned is not None and tuned["kernel"] in ("line", "point", "tensor")
    assert op.problem.device_errors() == 0
    orc = O.OracleProblem(V, Quadrature.gauss(4))
    orc.mf_prepare(x, V.dirichlet_values)
    assert reldiff(y.astype(np.float64), orc.mf_apply(dx.astype(np.float64))) < TOL32
