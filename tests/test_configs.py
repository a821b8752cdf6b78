"""GPU parity at the benchmark configurations' own sizes (not only on toy meshes).

* Assembly, the exact headline case: SVK (lambda = 2, mu = 1) on Q2 hexahedra 20 x 10 x 10, Gauss
  degree 4, x = 0 clamped and x = 1 displaced 0.05 on the faces' interiors (Gridap's face tags), the
  state u = 0.05 x e_x + U(-1e-3, 1e-3): colours, the CSC pattern and the positions bit-exact with the
  oracle (color_cells, src/coloring.jl:4-28; sparsity / cell_positions!, src/assembly.jl:773-899), the
  FP64 residual and CSC Jacobian within 1e-12 relative (jacobian!, src/assembly.jl:918-927), with the
  atomic and the colour-by-colour scatter. This is what the reference's own equality tests check
  against Gridap (test/test_gridap_equality.jl:18-36, test/test_assembly.jl:3-21). The element
  blocks are formed on the FP64 FMA pipe (default) and, once, on the FP64 tensor cores.
* Matrix-free product at sizes the oracle finishes in seconds: Q2 24^3 (338 541 free dofs) and Q4
  12^3 (the Q4 element of the Newton case): FP64 within 1e-12 of the oracle's stored-tangent mul!
  (src/matrixfree.jl:341-424), FP32 within 2e-6 of it. The FP32 error is printed and must be above
  FP64 round-off (the product really ran in single precision).
* Oseen P2-P1 on the 8^3 cube split into 3 072 tetrahedra with the outlet group: pattern bit-exact,
  residual and CSC Jacobian within 1e-12.
"""
import numpy as np
import pytest

from conftest import reldiff

import oracle as O
from hfk import forms
from hfk.fespace import CartesianMesh, Quadrature, VectorLagrangeSpace
from hfk.operator import KernelOperator, MatrixFreeJacobian

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-6


def _dirichlet():
    return [lambda x: 0 * x, lambda x: np.tile([0.05, 0.0, 0.0], (len(x), 1))]


def _state(V, seed=0):
    rng = np.random.default_rng(seed)
    x, _ = V.interpolate(lambda p: np.stack([0.05 * p[:, 0], 0 * p[:, 0], 0 * p[:, 0]], axis=1))
    return x + rng.uniform(-1e-3, 1e-3, V.nfree)


@pytest.fixture(scope="module")
def c0():
    V = VectorLagrangeSpace(CartesianMesh((20, 10, 10)), 2, ("x0", "x1"), g=_dirichlet(), open_faces=True)
    orc = O.OracleProblem(V, Quadrature.gauss(4))
    x = _state(V)
    return V, orc, x


def test_c0_sizes(c0):
    V, orc, x = c0
    # Q2 nodes 41 * 21 * 21, the open faces' interiors (2 * 19^2 nodes) fixed in 3 components
    assert V.mesh.ncells == 2000 and V.nfree == 52077 and V.ndir == 2166


def test_c0_colours_pattern_and_positions_bit_exact(c0):
    V, orc, x = c0
    op = KernelOperator(forms.svk_residual(2.0, 1.0, 4), forms.svk_jacobian(2.0, 1.0, 4), V)
    assert np.array_equal(op.problem.colors(), orc.colors)
    colptr, rowval = op.pattern_julia()
    ocp, orv = orc.pattern()
    assert len(orv) == 8990127
    assert np.array_equal(colptr, ocp) and np.array_equal(rowval, orv)
    assert np.array_equal(op.nonzero_positions(), orc.nzpos)


@pytest.mark.parametrize("scatter,kernel", [("atomic", "fma"), ("coloured", "fma"), ("atomic", "tensor")])
def test_c0_residual_and_jacobian_parity(c0, scatter, kernel):
    V, orc, x = c0
    op = KernelOperator(forms.svk_residual(2.0, 1.0, 4), forms.svk_jacobian(2.0, 1.0, 4), V)
    op.problem.set_scatter(scatter)
    op.problem.set_assembly_kernel(kernel)
    d = V.dirichlet_values
    b = op.residual(np.zeros(V.nfree), x)
    assert reldiff(b, orc.residual(x, d)) < TOL64
    A = op.allocate_jacobian(x)
    op.jacobian(A, x)
    ref = orc.jacobian_values(x, d)
    assert reldiff(A.data, ref) < TOL64
    # the second assembly into the same matrix zero-fills first
    op.jacobian(A, x)
    assert reldiff(A.data, ref) < TOL64


@pytest.mark.parametrize("order,n", [(2, 24), (4, 12)])
def test_c1_matrix_free_product_parity(order, n):
    V = VectorLagrangeSpace(CartesianMesh((n, n, n)), order, ("x0", "x1"), g=_dirichlet())
    deg = 2 * order
    op = KernelOperator(forms.svk_residual(2.0, 1.0, deg), forms.svk_jacobian(2.0, 1.0, deg), V, jacobian="matrixfree")
    orc = O.OracleProblem(V, Quadrature.gauss(deg))
    x = _state(V)
    dx = np.random.default_rng(1).standard_normal(V.nfree)
    orc.mf_prepare(x, V.dirichlet_values)
    ref = orc.mf_apply(dx)
    for mode in ("recompute", "stored"):
        mf = MatrixFreeJacobian(op, mode)
        op.jacobian(mf, x)
        assert reldiff(mf.mul(np.zeros(V.nfree), dx), ref) < TOL64, mode
    mf = MatrixFreeJacobian(op, "recompute")
    op.jacobian(mf, x)
    y32 = mf.mul_f32(np.zeros(V.nfree, dtype=np.float32), dx.astype(np.float32))
    err = reldiff(y32.astype(np.float64), ref)
    print(f"FP32 J*v Q{order} {n}^3: relative error vs the FP64 oracle {err:.2e}")
    assert 1e-12 < err < TOL32


@pytest.mark.parametrize("scatter", ["atomic", "coloured"])
def test_c2_oseen_assembly_parity(scatter):
    from hfk import oseen as OS

    m = OS.TetMesh(8)
    V = OS.TaylorHoodSpace(m)
    un, und = V.interpolate_velocity(OS.fourier_field(2))
    params = OS.OseenParams(rho=1.0, mu=1e-3, dt=1e-3, bdf2=True)
    op = OS.OseenOperator(V, params, un, und)
    op.set_outlet(OS.OutletFacets(m))
    op.set_scatter(scatter)
    orc = O.OracleOseen(V, params, un, und)
    orc.set_outlet(OS.OutletFacets(m))
    assert m.ncells == 3072
    A = op.sparsity_pattern()
    cp, rv = orc.pattern()
    assert np.array_equal(A.indptr, cp - 1) and np.array_equal(A.indices, rv - 1)
    assert reldiff(op.jacobian_values(np.zeros(A.nnz)), orc.jacobian_values()) < TOL64
    x = np.random.default_rng(0).standard_normal(V.nfree)
    d = V.dirichlet_values
    assert reldiff(op.residual(np.zeros(V.nfree), x, d), orc.residual(x, d)) < TOL64


def test_c0_jacobian_into_device_memory_repeatedly(c0):
    # device-resident state and values (the single-launch path of the persistent FMA kernel, the one
    # the benchmark times): five assemblies into the same array, with other values written in
    # between, all equal the oracle's (the zero-fill comes first every time)
    import torch

    from hfk import _lib

    V, orc, x = c0
    op = KernelOperator(forms.svk_residual(2.0, 1.0, 4), forms.svk_jacobian(2.0, 1.0, 4), V)
    nnz = op.sparsity_pattern().nnz
    ref = orc.jacobian_values(x, V.dirichlet_values)
    xd = torch.from_numpy(x).cuda()
    dd = torch.from_numpy(np.ascontiguousarray(V.dirichlet_values)).cuda()
    nz = torch.full((nnz,), 7.0, dtype=torch.float64, device="cuda")
    for k in range(5):
        _lib.call("hfk_jacobian", op.problem.h, _lib.ptr(xd), _lib.ptr(dd), _lib.ptr(nz))
        torch.cuda.synchronize()
        assert reldiff(nz.cpu().numpy(), ref) < TOL64, k
        nz.fill_(float(k + 1))
    assert op.problem.device_errors() == 0
