"""hfk: B200-native engine for HyperFEMKernels' hot path (Python host over the C ABI of libhfk.so).

The host side mirrors the reference's Julia API (``KernelOperator``, ``MatrixFreeJacobian``,
``MatrixFreeSolver``, ``PMultigrid``, ``Chebyshev``, ``BlockJacobi``, ``Prolongation``); every
numerical call runs CUDA kernels of ``libhfk.so``. ``fespace`` stands in for what Gridap supplies
(numbering, tables, Dirichlet data) on Cartesian hexahedral meshes.
"""
from . import fespace, forms
from .fespace import CartesianMesh, Quadrature, VectorLagrangeSpace, lagrange1d, transfer_matrices

__all__ = ["fespace", "forms", "CartesianMesh", "Quadrature", "VectorLagrangeSpace", "lagrange1d",
           "transfer_matrices", "KernelOperator", "MatrixFreeJacobian", "MatrixFreeSolver", "PMultigrid",
           "Chebyshev", "BlockJacobi", "Prolongation"]


def __getattr__(name):
    # the classes that call the library load it lazily, so that fespace/forms import without a GPU build
    import importlib

    if name in ("KernelOperator", "MatrixFreeJacobian", "Problem"):
        return getattr(importlib.import_module(__name__ + ".operator"), name)
    if name in ("MatrixFreeSolver", "PMultigrid", "Chebyshev", "BlockJacobi", "Prolongation", "chebyshev_damping",
                "eigenvalue_bounds"):
        return getattr(importlib.import_module(__name__ + ".solvers"), name)
    raise AttributeError(name)
