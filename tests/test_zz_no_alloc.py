"""The allocation-free smoother entry point (hfk_chebyshev_smooth_noalloc).

It serves callers that cannot allocate device memory once their solver is set up (a host that draws
every GPU buffer from a fixed pool, or an application that forbids allocation after set-up). Its
output must match the allocating entry point hfk_chebyshev_smooth, on two calls in a row (the
shared scratch array keeps the previous call's contents, so the second call checks that nothing
leaks from the first). This file is collected last, so a run that stops at the first failure has
already run every other test.
"""
import numpy as np
import pytest

from conftest import reldiff, svk_space, svk_state

from hfk import _lib, forms
from hfk._lib import call, ptr
from hfk.fespace import CartesianMesh, VectorLagrangeSpace
from hfk.operator import KernelOperator, MatrixFreeJacobian
from hfk import solvers as S

pytestmark = pytest.mark.gpu

TOL64 = 1e-12  # the FP64 tolerance of the parity tests


def _prepared_operator():
    V = svk_space(n=(3, 3, 2), order=2)
    op = KernelOperator(forms.svk_residual(2.0, 1.0, 4), forms.svk_jacobian(2.0, 1.0, 4), V, jacobian="matrixfree")
    x = svk_state(V, amp=1e-2)
    mf = MatrixFreeJacobian(op)
    op.jacobian(mf, x)
    st = S.BlockJacobiState(mf)
    assert st.ok
    lmin, lmax = S.eigenvalue_bounds(mf, st, 10)
    b = 1.1 * lmax
    return V, op, b / 20.0, b


def test_noalloc_smoother_matches_the_allocating_one_twice():
    import torch

    V, op, a, b = _prepared_operator()
    n = V.nfree
    rng = np.random.default_rng(7)
    rhs1 = torch.from_numpy(rng.standard_normal(n)).cuda()
    rhs2 = torch.from_numpy(rng.standard_normal(n)).cuda()
    h = op.problem.h
    x_ref = torch.zeros(n, dtype=torch.float64, device="cuda")
    r_ref = torch.zeros_like(x_ref)
    x_na = torch.zeros_like(x_ref)
    r_na = torch.zeros_like(x_ref)
    # first call: zero initial guess, with the residual
    call("hfk_chebyshev_smooth", h, a, b, 3, ptr(rhs1), ptr(x_ref), 1, ptr(r_ref))
    call("hfk_chebyshev_smooth_noalloc", h, a, b, 3, ptr(rhs1), ptr(x_na), 1, ptr(r_na))
    torch.cuda.synchronize()
    assert reldiff(x_na.cpu().numpy(), x_ref.cpu().numpy()) < TOL64
    assert reldiff(r_na.cpu().numpy(), r_ref.cpu().numpy()) < TOL64
    # second call in a row: the previous solution as initial guess, another right-hand side, no residual
    call("hfk_chebyshev_smooth", h, a, b, 4, ptr(rhs2), ptr(x_ref), 0, None)
    call("hfk_chebyshev_smooth_noalloc", h, a, b, 4, ptr(rhs2), ptr(x_na), 0, None)
    torch.cuda.synchronize()
    assert reldiff(x_na.cpu().numpy(), x_ref.cpu().numpy()) < TOL64
    assert float(torch.linalg.norm(x_na)) > 0


def test_noalloc_smoother_runs_no_autotuning():
    # a product that was never tuned stays untuned through the allocation-free call (the tuner's
    # candidate launches and host copies are not part of it); the default shape gives the same result
    import torch

    V = svk_space(n=(3, 3, 2), order=2)
    op = KernelOperator(forms.svk_residual(2.0, 1.0, 4), forms.svk_jacobian(2.0, 1.0, 4), V, jacobian="matrixfree")
    x0 = svk_state(V, amp=1e-2)
    mf = MatrixFreeJacobian(op)
    op.jacobian(mf, x0)
    st = S.BlockJacobiState(mf)
    assert st.ok
    assert op.problem.tuning("jv", "fp64") is None
    n = V.nfree
    rhs = torch.from_numpy(np.random.default_rng(8).standard_normal(n)).cuda()
    x_na = torch.zeros(n, dtype=torch.float64, device="cuda")
    x_ref = torch.zeros_like(x_na)
    call("hfk_chebyshev_smooth_noalloc", op.problem.h, 0.5, 10.0, 3, ptr(rhs), ptr(x_na), 1, None)
    torch.cuda.synchronize()
    assert op.problem.tuning("jv", "fp64") is None
    call("hfk_chebyshev_smooth", op.problem.h, 0.5, 10.0, 3, ptr(rhs), ptr(x_ref), 1, None)
    torch.cuda.synchronize()
    assert op.problem.tuning("jv", "fp64") is not None
    assert reldiff(x_na.cpu().numpy(), x_ref.cpu().numpy()) < TOL64


def test_noalloc_smoother_leaves_free_device_memory_unchanged():
    # the contract itself: after a first call (which resolves the scratch array's address), further
    # calls take no device memory
    import torch

    V, op, a, b = _prepared_operator()
    n = V.nfree
    rhs = torch.from_numpy(np.random.default_rng(3).standard_normal(n)).cuda()
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    r = torch.zeros_like(x)
    h = op.problem.h
    call("hfk_chebyshev_smooth_noalloc", h, a, b, 3, ptr(rhs), ptr(x), 1, ptr(r))
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for k in range(5):
        call("hfk_chebyshev_smooth_noalloc", h, a, b, 2 + k % 3, ptr(rhs), ptr(x), 0, ptr(r))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_smoother_rejects_host_pointers_and_too_many_dofs():
    V, op, a, b = _prepared_operator()
    rhs = np.ones(V.nfree)
    x = np.zeros(V.nfree)
    with pytest.raises(_lib.HFKError) as e:
        call("hfk_chebyshev_smooth_noalloc", op.problem.h, a, b, 2, ptr(rhs), ptr(x), 1, None)
    assert "device pointers" in str(e.value)
    # Q1 on a 64^3 mesh: 823 875 nodes, beyond the stated maximum of free dofs
    m = CartesianMesh((64, 64, 64))
    big = VectorLagrangeSpace(m, 1, ("x0", "x1"))
    assert big.nfree > 524288
    opb = KernelOperator(forms.svk_residual(2.0, 1.0, 2), forms.svk_jacobian(2.0, 1.0, 2), big)
    import torch

    r = torch.ones(big.nfree, dtype=torch.float64, device="cuda")
    y = torch.zeros_like(r)
    with pytest.raises(_lib.HFKError) as e:
        call("hfk_chebyshev_smooth_noalloc", opb.problem.h, a, b, 2, ptr(r), ptr(y), 1, None)
    assert e.value.code == 1 and "at most 524288 free dofs" in str(e.value)
    # vectors on another GPU than the operator's (needs two GPUs)
    if torch.cuda.device_count() > 1:
        r1 = torch.ones(V.nfree, dtype=torch.float64, device="cuda:1")
        x1 = torch.zeros_like(r1)
        with pytest.raises(_lib.HFKError) as e:
            call("hfk_chebyshev_smooth_noalloc", op.problem.h, a, b, 2, ptr(r1), ptr(x1), 1, None)
        assert "operator's GPU" in str(e.value)
