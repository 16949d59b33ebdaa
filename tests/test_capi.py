"""The C-ABI library loads, exports every declared symbol and reports errors."""
from __future__ import annotations

import ctypes
import os

import numpy as np

from tensors_b200 import _lib
from tensors_b200.cholesky import CholeskyDecomposition, TBError


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    declared = _lib.declared_symbols()
    assert len(declared) >= 30
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    # and the Python binding covers them all
    assert set(declared) <= set(_lib.SIGNATURES)


def test_library_is_built_for_sm100a():
    # the kernels are compiled for sm_100a only (build.py GENCODE)
    from tensors_b200 import build

    assert build.GENCODE == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert os.path.exists(_lib.LIB_PATH)


def test_error_paths_without_a_device():
    lib = _lib.lib()
    h = ctypes.c_void_p()
    outer = np.array([0, 1], dtype=np.int64)
    inner = np.array([0], dtype=np.int32)
    assert lib.tb_chol_create(ctypes.byref(h), 0, outer.ctypes.data, inner.ctypes.data, None, 1) == -1
    assert b"n of matrix" in lib.tb_last_error()
    assert lib.tb_chol_symbolic(None) == -1
    assert lib.tb_chol_set_supernode_strategy(None, 0) == -1
    c = CholeskyDecomposition(outer, inner)
    # solving before factorizing is an error (Solve.hpp:353-363)
    try:
        c.Solve(np.ones(1))
        raise AssertionError("expected TBError")
    except TBError as e:
        assert e.status == -5
    assert not c.NumericallyFactorizedQ()
