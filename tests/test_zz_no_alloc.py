"""tb_chol_solve_device_noalloc: the solve whose work block is a fixed device
array, for callers that may not allocate device memory at solve time.  Called
through the C-ABI and compared with tb_chol_solve_device on the same
factorization, twice in a row (the second call reuses the array without any
set-up); more right-hand sides than one sweep chunk takes; two handles solved
in turn through the one shared array; refining handles are turned away."""
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


def _factored(grid, seed, shift, precision="fp64"):
    A = matrices.grid_laplacian_3d(grid, seed, shift)
    chol = CholeskyDecomposition(A.outer, A.inner, ordering.nested_dissection(A))
    chol.SetPrecision(precision)
    chol.SymbolicFactorization()
    assert chol.NumericFactorization(A.values, 0.0) == 0
    return A, chol


def _both(lib, chol, B, k):
    import torch

    X_ref = torch.zeros_like(B)
    assert lib.tb_chol_solve_device(chol.handle, 1.0, B.data_ptr(), k, 0.0, X_ref.data_ptr(), k, k) == 0
    X = torch.full_like(B, float("nan"))
    assert lib.tb_chol_solve_device_noalloc(chol.handle, 1.0, B.data_ptr(), k, 0.0, X.data_ptr(), k, k) == 0, \
        lib.tb_last_error()
    torch.cuda.synchronize()
    return X, X_ref


@pytest.mark.gpu
def test_noalloc_solve_more_rhs_than_one_sweep_chunk():
    """70 right-hand sides: the sweeps take them as a 64-wide and a 6-wide chunk inside the fixed array."""
    import torch

    A, chol = _factored(12, 0x5EED0022, 1e-3)
    k = 70
    assert A.n * k <= SCRATCH_ENTRIES
    B = torch.tensor(np.random.default_rng(23).standard_normal((A.n, k)), device="cuda")
    lib = _lib.lib()
    for _ in range(2):
        X, X_ref = _both(lib, chol, B, k)
        assert float(torch.linalg.norm(X - X_ref)) <= 1e-12 * float(torch.linalg.norm(X_ref))


@pytest.mark.gpu
def test_noalloc_two_handles_in_turn_share_the_array():
    """Two handles of different sizes solved one after the other: each result equals its own device solve."""
    import torch

    lib = _lib.lib()
    cases = [_factored(10, 0x5EED0024, 1e-2), _factored(13, 0x5EED0025, 1e-4)]
    Bs = [torch.tensor(np.random.default_rng(24 + i).standard_normal((A.n, 3 + i)), device="cuda")
          for i, (A, _) in enumerate(cases)]
    for _ in range(2):
        for (A, chol), B in zip(cases, Bs):
            X, X_ref = _both(lib, chol, B, B.shape[1])
            assert float(torch.linalg.norm(X - X_ref)) <= 1e-12 * float(torch.linalg.norm(X_ref))


@pytest.mark.gpu
def test_noalloc_solve_turns_away_refining_handles():
    """A mixed-precision handle is solved by refinement, which needs more work vectors than the fixed array
    holds: the call fails with a status and leaves X untouched."""
    import torch

    A, chol = _factored(10, 0x5EED0026, 1e-2, precision="mixed")
    k = 2
    B = torch.ones((A.n, k), dtype=torch.float64, device="cuda")
    X = torch.full_like(B, 7.0)
    lib = _lib.lib()
    dev_before = torch.cuda.current_device()
    rc = lib.tb_chol_solve_device_noalloc(chol.handle, 1.0, B.data_ptr(), k, 0.0, X.data_ptr(), k, k)
    assert rc == -1
    assert b"refinement" in lib.tb_last_error()
    torch.cuda.synchronize()
    assert bool((X == 7.0).all())
    assert torch.cuda.current_device() == dev_before
