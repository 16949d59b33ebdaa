"""MatrixMarket coordinate files <-> CSR, through the library's host reader and writer.

Mirrors ``MatrixCSR::LoadFromMatrixMarket`` and ``MatrixCSR::WriteToMatrixMarket``
(src/Sparse/MatrixCSR/MatrixMarket.hpp:3-202, :205-306): fields real, integer and
pattern, symmetry general and symmetric (the stored triangle is mirrored, the
diagonal kept once), columns sorted per row and repeated entries summed in file
order (``MatrixCSR::FromTriples``, src/Sparse/MatrixCSR/FromTriples.hpp:4-209).
Failures raise :class:`~tensors_b200.cholesky.TBError` with ``TB_ERR_IO`` (-11)
or ``TB_ERR_FORMAT`` (-12).  The parse runs in native code on all host threads.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from ._lib import lib
from .cholesky import _check
from .matrices import CSRMatrix

__all__ = ["read_matrix_market", "load_matrix_market", "write_matrix_market"]


def read_matrix_market(path, thread_count: int = 0):
    """(rows, cols, outer int64[rows+1], inner int32[nnz], values float64[nnz]) of a coordinate file."""
    L = lib()
    rows, cols = ctypes.c_int32(), ctypes.c_int32()
    po = ctypes.POINTER(ctypes.c_int64)()
    pi = ctypes.POINTER(ctypes.c_int32)()
    pv = ctypes.POINTER(ctypes.c_double)()
    _check(L.tb_matrix_market_read(os.fsencode(path), int(thread_count), ctypes.byref(rows), ctypes.byref(cols),
                                   ctypes.byref(po), ctypes.byref(pi), ctypes.byref(pv)))
    try:
        m = rows.value
        outer = np.ctypeslib.as_array(po, shape=(m + 1,)).copy()
        nnz = int(outer[-1])
        inner = np.ctypeslib.as_array(pi, shape=(max(nnz, 1),))[:nnz].copy()
        values = np.ctypeslib.as_array(pv, shape=(max(nnz, 1),))[:nnz].copy()
    finally:
        for p in (po, pi, pv):
            L.tb_matrix_market_free(ctypes.cast(p, ctypes.c_void_p))
    return m, cols.value, outer, inner, values


def load_matrix_market(path, thread_count: int = 0) -> CSRMatrix:
    """A square coordinate file as the :class:`CSRMatrix` the Cholesky path consumes."""
    m, n, outer, inner, values = read_matrix_market(path, thread_count)
    if m != n:
        raise ValueError(f"{path}: {m} x {n} matrix is not square")
    return CSRMatrix(n=m, outer=outer, inner=inner, values=values)


def write_matrix_market(path, A, cols: int | None = None) -> None:
    """Write a :class:`CSRMatrix` (or ``(rows, outer, inner, values)``) as a real general coordinate file."""
    if isinstance(A, CSRMatrix):
        rows, outer, inner, values = A.n, A.outer, A.inner, A.values
    else:
        rows, outer, inner, values = A
    cols = rows if cols is None else cols
    outer = np.ascontiguousarray(outer, dtype=np.int64)
    inner = np.ascontiguousarray(inner, dtype=np.int32)
    values = np.ascontiguousarray(values, dtype=np.float64)
    if outer.shape != (rows + 1,) or inner.shape != values.shape or len(inner) != int(outer[-1]):
        raise ValueError("write_matrix_market: inconsistent CSR arrays")
    _check(lib().tb_matrix_market_write(os.fsencode(path), int(rows), int(cols), outer.ctypes.data,
                                        inner.ctypes.data, values.ctypes.data))
