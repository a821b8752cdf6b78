"""The C ABI library loads and exports every symbol that include/hfk.h declares (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, has_gpu

from hfk import _lib


def declared_functions():
    src = open(os.path.join(ROOT, "include", "hfk.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(hfk_[a-z0-9_]+)\s*\(", src)))


def test_every_declared_symbol_is_exported_and_bound():
    L = _lib.lib()
    names = declared_functions()
    assert len(names) >= 30
    for n in names:
        assert hasattr(L, n), n
        assert n in _lib.SIGNATURES or n == "hfk_last_error", f"{n} has no ctypes signature"


def test_version_and_error_prefix():
    L = _lib.lib()
    assert L.hfk_version() >= 100
    with pytest.raises(_lib.HFKError) as e:
        _lib.call("hfk_problem_create", None, 0, 0, 0, 0, None, None, None, None, None, None, None, 0, 0, 1, None, 0)
    assert str(e.value).startswith("HyperFEMKernels: ")
    assert e.value.code == 1


def test_hessenberg_eigenvalues_match_lapack():
    # the eigvals call of eigenvalue_bounds (src/preconditioners.jl:386) in the library's host code
    from hfk.solvers import hessenberg_eigvals

    rng = np.random.default_rng(0)
    for n in (1, 2, 3, 5, 10, 20):
        for sym in (False, True):
            A = rng.standard_normal((n, n))
            if sym:
                A = A @ A.T + n * np.eye(n)
            H = np.triu(A, -1)
            ev = np.sort_complex(hessenberg_eigvals(H))
            ref = np.sort_complex(np.linalg.eigvals(H))
            assert np.allclose(ev, ref, atol=1e-9 * max(1, np.abs(ref).max())), (n, ev, ref)


@pytest.mark.skipif(has_gpu(), reason="checks the failure mode without a GPU")
def test_operations_fail_loudly_without_a_device():
    from conftest import svk_space
    from hfk.forms import svk_residual, svk_jacobian
    from hfk.operator import KernelOperator

    V = svk_space(order=2)
    with pytest.raises(_lib.HFKError) as e:
        KernelOperator(svk_residual(), svk_jacobian(), V)
    assert "CUDA" in str(e.value)


def test_set_tolerance_is_the_forcing_term_hook():
    # test/solvers/test_matrixfree_solver.jl:75-92 (the host side of it: the solve itself is on the GPU)
    import types

    from hfk import solvers as S

    ns = types.SimpleNamespace(solver=S.MatrixFreeSolver(rtol=1e-10), rtol=1e-10)
    assert S.tolerance(ns) == 1e-10
    S.set_tolerance(ns, 1e-2)
    assert S.tolerance(ns) == 1e-2
    S.set_tolerance(ns, None)
    assert S.tolerance(ns) == 1e-10
    with pytest.raises(ValueError, match="HyperFEMKernels"):
        S.set_tolerance(ns, 1.5)


def test_solver_options_are_validated_before_any_device_work():
    # test/solvers/test_matrixfree_solver.jl:55-73, test/solvers/test_operator.jl:89-95,
    # test/solvers/test_pmultigrid_levels.jl:143 (the option checks; the GPU parts run in the gpu tests)
    from hfk import forms
    from hfk import solvers as S
    from hfk.fespace import CartesianMesh, VectorLagrangeSpace
    from hfk.operator import KernelOperator

    for bad in (dict(krylov="bicgstab"), dict(restart=0), dict(rtol=1.0), dict(rtol=-1e-3), dict(atol=-1.0),
                dict(maxiter=0)):
        with pytest.raises(ValueError, match="HyperFEMKernels"):
            S.MatrixFreeSolver(**bad)
    m = CartesianMesh((2, 2, 2))
    Vs = [VectorLagrangeSpace(m, o, ("x0",)) for o in (2, 1)]
    for args, kw in (((Vs[:1],), {}), ((Vs,), dict(coarse_every=0)), ((Vs,), dict(precision="fp16")),
                     ((Vs,), dict(coarse="amg")), ((Vs,), dict(coarse="cg", coarse_iters=0))):
        with pytest.raises(ValueError, match="HyperFEMKernels"):
            S.PMultigrid(*args, **kw)
    for kw in (dict(solver="lu"), dict(every=0)):
        with pytest.raises(ValueError, match="HyperFEMKernels"):
            S.LaggedAssembled(**kw)
    res, jac = forms.svk_residual(), forms.svk_jacobian()
    with pytest.raises(ValueError, match="HyperFEMKernels"):
        KernelOperator(res, jac, Vs[0], jacobian="dense")
    with pytest.raises(ValueError, match="HyperFEMKernels"):
        KernelOperator(res, forms.svk_jacobian(lam=3.0), Vs[0])  # residual and Jacobian of different laws


def test_pointer_keeps_a_temporary_alive():
    # ptr() of a temporary copy: the pointer object must keep the copy alive until the call that
    # receives it returns (the outlet normals are passed as np.asfortranarray(...) in place)
    import gc

    from hfk._lib import ptr

    a = np.arange(12.0).reshape(3, 4)
    p = ptr(np.asfortranarray(a))
    gc.collect()
    junk = [np.full(12, -1.0) for _ in range(64)]  # would reuse a freed block
    view = np.ctypeslib.as_array(ctypes.cast(p, ctypes.POINTER(ctypes.c_double)), shape=(12,))
    assert np.array_equal(view, np.asfortranarray(a).ravel(order="K")) and len(junk) == 64


def test_problem_outlives_its_hierarchies_whatever_the_finalisation_order(monkeypatch):
    # a hierarchy reads its level problems when destroyed: a problem whose owner is finalised first
    # (cyclic garbage is finalised in no particular order) is destroyed with the last hierarchy
    destroyed = []

    class FakeLib:
        def hfk_problem_destroy(self, h):
            destroyed.append(h.value)

    monkeypatch.setattr(_lib, "lib", lambda: FakeLib())
    _lib.retain_problem(11)
    _lib.retain_problem(11)
    _lib.retain_problem(12)
    _lib.destroy_problem(11)  # owner gone, two hierarchies still use it
    _lib.destroy_problem(13)  # used by none: destroyed at once
    assert destroyed == [13]
    _lib.release_problem(11)
    assert destroyed == [13]
    _lib.release_problem(12)  # its owner is still alive: nothing destroyed
    _lib.release_problem(11)  # the last user of 11
    assert destroyed == [13, 11]
    _lib.destroy_problem(12)
    assert destroyed == [13, 11, 12] and not _lib._users and not _lib._pending
