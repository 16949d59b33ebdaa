"""B200-native supernodal sparse Cholesky factor-and-solve.

A drop-in for the ``Sparse::CholeskyDecomposition`` path of
HenrikSchumacher/Tensors: host-side symbolic analysis in C++ and the numeric
factorization and multi-RHS solves as hand-written sm_100a CUDA kernels,
reached through the C-ABI declared in ``include/tensors_b200.h``.
"""
from . import matrices, ordering  # noqa: F401

# the library-backed modules (cholesky, serving, matrix_market) load the shared
# object on first use: ``from tensors_b200.cholesky import CholeskyDecomposition``
__all__ = ["matrices", "ordering", "cholesky", "serving", "matrix_market"]
