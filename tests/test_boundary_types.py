"""The boundary's scalar types and the numeric-factor container.

* ``NumericFactorization<ExtScal>`` (Numeric.hpp:3-8): float32 values are
  converted to FP64 on copy, so they factor exactly like their FP64 images.
* ``Solve`` with B and X of either type (Solve.hpp:20-27, cast on copy):
  float32 right-hand sides solve like their FP64 images, a float32 X
  receives the FP64 solution rounded once; a float-in / double-out solve
  matches the oracle.  Two solves of one system agree to FP64 rounding, not
  bit for bit: the sweeps add contributions into ancestor rows with atomic
  additions, in no fixed order.
* ``NumericalFactorization_T`` + ``SwapNumericalFactorization``
  (CholeskyDecomposition.hpp:132-201, Numeric.hpp:228-254): factors move
  between decompositions of one pattern and keep solving their own matrix; a
  factor too small for the receiving symbolic analysis arrives unfactorized;
  a mixed-precision factor brings its precision along.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from tensors_b200 import matrices as M
from tensors_b200 import ordering as O
from tensors_b200.cholesky import CholeskyDecomposition, NumericalFactorization, TBError

pytestmark = pytest.mark.gpu


def _system(seed=0x5EED0031, g=12):
    A = M.grid_laplacian_3d(g, seed, 1e-2)
    return A, O.nested_dissection(A)


def test_float32_values_factor_like_their_fp64_image():
    A, perm = _system()
    v32 = A.values.astype(np.float32)
    c32 = CholeskyDecomposition(A.outer, A.inner, perm)
    c64 = CholeskyDecomposition(A.outer, A.inner, perm)
    assert c32.NumericFactorization(v32, 0.0) == 0
    assert c64.NumericFactorization(v32.astype(np.float64), 0.0) == 0
    t32, r32 = c32.FactorValues()
    t64, r64 = c64.FactorValues()
    assert np.array_equal(t32, t64) and np.array_equal(r32, r64)


def close(X, Y, tol=1e-13):
    X, Y = np.asarray(X, dtype=np.float64), np.asarray(Y, dtype=np.float64)
    return float(np.abs(X - Y).max() / np.abs(Y).max()) < tol


def test_solve_casts_right_hand_sides_and_solutions_on_copy():
    A, perm = _system()
    c = CholeskyDecomposition(A.outer, A.inner, perm)
    assert c.NumericFactorization(A.values, 0.0) == 0
    B32 = np.random.default_rng(31).standard_normal((A.n, 5)).astype(np.float32)
    X64 = c.Solve(B32.astype(np.float64))
    # float in, double out: the same solve as the FP64 image of B
    Xa = np.zeros((A.n, 5), dtype=np.float64)
    c.Solve(B32, Xa)
    assert close(Xa, X64)
    # double in, float out: the FP64 solution rounded once (one float32 ulp)
    Xb = np.zeros((A.n, 5), dtype=np.float32)
    c.Solve(B32.astype(np.float64), Xb)
    assert np.all(np.abs(Xb.astype(np.float64) - X64) <= 1.2e-7 * np.abs(X64) + 1e-30)
    # float in, float out, with alpha / beta on a float X
    X0 = np.random.default_rng(32).standard_normal((A.n, 5)).astype(np.float32)
    Xc = X0.copy()
    c.Solve(B32, Xc, alpha=2.0, beta=-0.5)
    E = 2.0 * X64 - 0.5 * X0.astype(np.float64)
    assert np.all(np.abs(Xc.astype(np.float64) - E) <= 1.2e-7 * np.abs(E) + 1e-12 * np.abs(E).max())
    # the float-in / double-out solve against the oracle
    ref = oracle.OracleCholesky(A.n, A.outer, A.inner, perm)
    assert ref.factor(A.values, 0.0) == 0
    Xo = ref.solve(B32.astype(np.float64))
    assert np.abs(Xa - Xo).max() / np.abs(Xo).max() < 1e-10


def test_device_solve_and_values_in_float32():
    import torch

    A, perm = _system()
    c = CholeskyDecomposition(A.outer, A.inner, perm)
    assert c.NumericFactorization(torch.tensor(A.values.astype(np.float32), device="cuda"), 0.0) == 0
    ref = CholeskyDecomposition(A.outer, A.inner, perm)
    assert ref.NumericFactorization(A.values.astype(np.float32).astype(np.float64), 0.0) == 0
    B = torch.tensor(np.random.default_rng(33).standard_normal((A.n, 3)), device="cuda")
    X64 = ref.Solve(B)
    X32 = c.Solve(B.float())                                  # float in, float out
    torch.cuda.synchronize()
    assert X32.dtype == torch.float32
    Xw = c.Solve(B.float(), torch.empty_like(B))             # float in, double out
    Xr = ref.Solve(B.float().double())
    assert close(Xw.cpu().numpy(), Xr.cpu().numpy())
    assert close(X32.cpu().numpy(), Xr.cpu().numpy(), 1e-6)
    assert float((X32.double() - X64).abs().max() / X64.abs().max()) < 1e-6


def test_swap_moves_factors_between_decompositions():
    A, perm = _system()
    A2 = M.grid_laplacian_3d(12, 0x5EED0032, 1e-2)          # same pattern, other values
    assert np.array_equal(A.outer, A2.outer) and np.array_equal(A.inner, A2.inner)
    h1 = CholeskyDecomposition(A.outer, A.inner, perm)
    h2 = CholeskyDecomposition(A.outer, A.inner, perm)
    assert h1.NumericFactorization(A.values, 0.0) == 0
    assert h2.NumericFactorization(A2.values, 0.0) == 0
    B = np.random.default_rng(34).standard_normal((A.n, 2))
    X1, X2 = h1.Solve(B), h2.Solve(B)                     # also captures the solve graphs
    f = NumericalFactorization()
    assert not f.NumericallyFactorizedQ() and f.AllocatedByteCount() == 0
    h1.SwapNumericalFactorization(f)                      # h1 <- empty, f <- A's factor
    assert f.NumericallyFactorizedQ() and f.NumericallyGoodQ() and f.AllocatedByteCount() > 0
    assert not h1.NumericallyFactorizedQ()
    with pytest.raises(TBError):
        h1.Solve(B)
    h2.SwapNumericalFactorization(f)                      # h2 <- A's factor, f <- A2's
    assert close(h2.Solve(B), X1)
    h1.SwapNumericalFactorization(f)                      # h1 <- A2's factor, f <- empty
    assert close(h1.Solve(B), X2)
    assert not f.NumericallyFactorizedQ()
    assert not close(X1, X2, 1e-3)                        # the two systems do differ
    # a factorization after a swap runs on the storage the handle now holds
    assert h2.NumericFactorization(A2.values, 0.0) == 0
    assert close(h2.Solve(B), X2)


def test_swap_into_a_decomposition_that_never_factored():
    A, perm = _system()
    h1 = CholeskyDecomposition(A.outer, A.inner, perm)
    assert h1.NumericFactorization(A.values, 0.0) == 0
    B = np.random.default_rng(37).standard_normal((A.n, 4))
    X1 = h1.Solve(B)
    f = NumericalFactorization()
    h1.SwapNumericalFactorization(f)
    fresh = CholeskyDecomposition(A.outer, A.inner, perm)    # no symbolic phase, no device plan yet
    fresh.SwapNumericalFactorization(f)
    assert fresh.NumericallyFactorizedQ()
    assert close(fresh.Solve(B), X1)


def test_swap_treats_a_too_small_factor_as_unfactorized():
    small, ps = _system(g=6)
    big, pb = _system(g=12)
    hs = CholeskyDecomposition(small.outer, small.inner, ps)
    hb = CholeskyDecomposition(big.outer, big.inner, pb)
    assert hs.NumericFactorization(small.values, 0.0) == 0
    assert hb.NumericFactorization(big.values, 0.0) == 0
    f = NumericalFactorization()
    hs.SwapNumericalFactorization(f)                      # f <- the small factor
    hb.SwapNumericalFactorization(f)                      # hb <- the small factor: too small
    assert not hb.NumericallyFactorizedQ()
    # the big handle factors again on storage grown to its size
    assert hb.NumericFactorization(big.values, 0.0) == 0
    B = np.random.default_rng(35).standard_normal(big.n)
    X = hb.Solve(B)
    S = big.to_scipy()
    assert np.linalg.norm(B - S @ X) / np.linalg.norm(B) < 1e-12


def test_swap_brings_the_mixed_precision_factor_along():
    A, perm = _system()
    hm = CholeskyDecomposition(A.outer, A.inner, perm)
    hm.SetPrecision("mixed")
    hm.SetRefinement(1e-12, 30)
    assert hm.NumericFactorization(A.values, 0.0) == 0
    hd = CholeskyDecomposition(A.outer, A.inner, perm)
    hd.SetRefinement(1e-12, 30)
    assert hd.NumericFactorization(A.values, 0.0) == 0
    f = NumericalFactorization()
    hm.SwapNumericalFactorization(f)
    assert f.Precision() == "mixed"
    hd.SwapNumericalFactorization(f)                      # hd <- the mixed factor, f <- the FP64 one
    assert hd.PrecisionInUse()[0] == "mixed" and f.Precision() == "fp64"
    B = np.random.default_rng(36).standard_normal((A.n, 3))
    X = hd.Solve(B)
    S = A.to_scipy()
    assert np.linalg.norm(B - S @ X) / np.linalg.norm(B) <= 1e-12
