"""B200 (sm_100a) implementation of the sparse solver path of nickreserved/CompressionTests.

CSR and DuVi sparse matrix-vector products, weighted Jacobi and Gauss-Seidel
smoothing, geometric-multigrid transfers and the PCG reductions, behind the C
ABI of include/duvi_gpu.h (libduvigpu.so, built in-tree).  This package is a
thin Python view of that ABI, shaped like the reference's C# solver classes.
"""
from . import _native
from ._native import DuviError, NotImplementedFeatureError, NotInitializedError, NoDeviceError
from .sparse import CudaContext, SparseMatrix
from .adjoint import AdjointCantilever, cantilever_solve_function, element_gradient_device
from .solvers import (CudaCsrGeometricMultigridSolver, CudaCsrPcgSolver, CudaDuViGeometricMultigridSolver,
                      BatchedMultigridSolver, IterativeStatistics, MultigridPcgSolver, make_path)
from .cantilever import (FemCantilever3D, cantilever_batch, cartesian_transfer, duvi_encode, galerkin,
                         galerkin_hierarchy, hex_assemble_device, hex_csr_size, hex_hierarchy, hex_stiffness,
                         hex_trilinear, random_face_loads,
                         traction_rhs, units_decode, units_encode)

__all__ = [
    "AdjointCantilever", "cantilever_solve_function", "element_gradient_device",
    "CudaContext", "SparseMatrix", "CudaCsrGeometricMultigridSolver", "CudaDuViGeometricMultigridSolver",
    "CudaCsrPcgSolver", "MultigridPcgSolver", "BatchedMultigridSolver", "cantilever_batch", "IterativeStatistics", "FemCantilever3D", "hex_hierarchy",
    "hex_stiffness", "hex_assemble_device", "hex_csr_size", "hex_trilinear", "duvi_encode", "units_encode", "units_decode", "galerkin", "galerkin_hierarchy", "traction_rhs", "random_face_loads", "cartesian_transfer", "make_path", "DuviError",
    "NotImplementedFeatureError", "NotInitializedError", "NoDeviceError",
]


def load():
    """Load the native library now (raises ImportError if it was not built)."""
    return _native.lib()
