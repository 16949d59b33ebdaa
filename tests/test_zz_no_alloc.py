"""tb_chol_solve_device_noalloc: the solve whose work block is a fixed device
array.  Called through the C-ABI and compared with tb_chol_solve_device on
the same factorization, twice in a row (the second call reuses the array
without any set-up)."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from tensors_b200 import _lib, matrices, ordering
from tensors_b200.cholesky import CholeskyDecomposition

SCRATCH_ENTRIES = 1 << 22


@pytest.mark.gpu
def test_noalloc_solve_matches_solve_device():
    import torch

    A = matrices.grid_laplacian_3d(14, 0x5EED0021, 1e-3)
    perm = ordering.nested_dissection(A)
    chol = CholeskyDecomposition(A.outer, A.inner, perm)
    chol.SymbolicFactorization()
    assert chol.NumericFactorization(A.values, 0.0) == 0
    lib = _lib.lib()
    h = chol.handle
    k = 5
    B = torch.tensor(np.random.default_rng(21).standard_normal((A.n, k)), device="cuda")
    X_ref = torch.zeros_like(B)
    assert lib.tb_chol_solve_device(h, 1.0, B.data_ptr(), k, 0.0, X_ref.data_ptr(), k, k) == 0
    torch.cuda.synchronize()
    tol = 1e-12 * float(torch.linalg.norm(X_ref))
    for _ in range(2):
        X = torch.full_like(B, float("nan"))
        assert lib.tb_chol_solve_device_noalloc(h, 1.0, B.data_ptr(), k, 0.0, X.data_ptr(), k, k) == 0, \
            lib.tb_last_error()
        torch.cuda.synchronize()
        assert float(torch.linalg.norm(X - X_ref)) <= tol
    # alpha / beta with a wider leading dimension of X
    X0 = torch.tensor(np.random.default_rng(22).standard_normal((A.n, k + 3)), device="cuda")
    X = X0.clone()
    assert lib.tb_chol_solve_device_noalloc(h, 2.0, B.data_ptr(), k, -0.5, X.data_ptr(), k + 3, k) == 0
    torch.cuda.synchronize()
    expect = 2.0 * X_ref - 0.5 * X0[:, :k]
    assert float(torch.linalg.norm(X[:, :k] - expect)) <= 4 * tol
    assert torch.equal(X[:, k:], X0[:, k:])


@pytest.mark.gpu
def test_noalloc_solve_rejects_requests_beyond_the_fixed_scratch():
    import torch

    A = matrices.grid_laplacian_2d(64, 1e-2)
    chol = CholeskyDecomposition(A.outer, A.inner, ordering.nested_dissection(A))
    chol.SymbolicFactorization()
    assert chol.NumericFactorization(A.values, 0.0) == 0
    k = SCRATCH_ENTRIES // A.n + 1
    B = torch.zeros((A.n, k), dtype=torch.float64, device="cuda")
    X = torch.zeros_like(B)
    lib = _lib.lib()
    rc = lib.tb_chol_solve_device_noalloc(chol.handle, 1.0, B.data_ptr(), k, 0.0, X.data_ptr(), k, k)
    assert rc == -1
    assert b"exceeds the fixed scratch" in lib.tb_last_error()
