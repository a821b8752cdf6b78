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
    if name in ("KernelOperator", "MatrixFreeJacobian", "Problem"):
        from . import operator

        return getattr(operator, name)
    if name in ("MatrixFreeSolver", "PMultigrid", "Chebyshev", "BlockJacobi", "Prolongation", "solvers",
                "chebyshev_damping", "eigenvalue_bounds"):
        from . import solvers

        return solvers if name == "solvers" else getattr(solvers, name)
    raise AttributeError(name)
