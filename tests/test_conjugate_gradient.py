"""Conjugate gradients preconditioned by the GPU factor (tb_chol_cg / _device).

Checked against a numpy restatement of the reference's
``ConjugateGradient::operator()`` (ConjugateGradient.hpp:109-356) whose
preconditioner is the oracle's factor solve: the same iteration counts (to one
step: summation order differs), solutions whose true residuals meet the
target, and the reference's argument semantics (alpha / beta, initial guess,
zero right-hand side, iteration cap).
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from tensors_b200 import matrices as M
from tensors_b200 import ordering as O
from tensors_b200.cholesky import CholeskyDecomposition

pytestmark = pytest.mark.gpu


def _cg_restatement(A, P, B, tol, max_iter, X0=None):
    """ConjugateGradient.hpp:164-343 with the operator A (CSR) and preconditioner P (a callable)."""
    r = B.copy()
    z = P(r)
    bsq = np.abs(np.sum(r * z, axis=0))
    TOL = bsq * tol * tol
    x = np.zeros_like(B)
    if X0 is not None:
        x = X0.copy()
        r = r - M.csr_matvec(A, x)
        z = P(r)
    p = z.copy()
    rho = np.sum(r * z, axis=0)
    it = 0
    while not np.all(np.abs(rho) <= TOL) and it < max_iter:
        u = M.csr_matvec(A, p)
        alpha = rho / np.sum(p * u, axis=0)
        x = x + alpha * p
        r = r - alpha * u
        z = P(r)
        rho_old, rho = rho, np.sum(r * z, axis=0)
        p = z + (rho / rho_old) * p
        it += 1
    return x, it, np.sqrt(np.abs(rho) / bsq)


def _nearby_pair(g=20):
    """A and A' = D A D with D = diag(1 + 0.1 u), u ~ U[-1, 1]: same pattern, SPD, nearby."""
    A = M.grid_laplacian_3d(g, 31, 1e-3)           # factored
    d = 1.0 + 0.1 * np.random.default_rng(32).uniform(-1.0, 1.0, A.n)
    rows = np.repeat(np.arange(A.n), np.diff(A.outer))
    A2 = M.CSRMatrix(n=A.n, outer=A.outer, inner=A.inner, values=d[rows] * A.values * d[A.inner])
    return A, A2, O.nested_dissection(A, 16)


def _relres(A, X, B):
    return np.linalg.norm(B - M.csr_matvec(A, X)) / np.linalg.norm(B)


def test_cg_on_a_nearby_matrix_matches_the_restatement():
    A, A2, perm = _nearby_pair()
    c = CholeskyDecomposition(A.outer, A.inner, perm)
    assert c.NumericFactorization(A.values) == 0
    o = oracle.OracleCholesky(A.n, A.outer, A.inner, perm)
    assert o.factor(A.values) == 0
    B = np.random.default_rng(2).standard_normal((A.n, 4))
    X, ok = c.ConjugateGradient(B, values=A2.values, relative_tolerance=1e-12, max_iter=300)
    assert ok
    x_ref, it_ref, rel_ref = _cg_restatement(A2, lambda R: o.solve(R), B, 1e-12, 300)
    # same recurrence, other summation order: the step counts agree to rounding
    assert abs(c.IterationCount() - it_ref) <= max(1, it_ref // 10) and it_ref > 3
    assert np.all(c.RelativeResiduals() <= 1e-12)
    # the criterion is in the P-norm: |r| / |b| <= sqrt(cond(A)) * 1e-12, cond(A) < 1e6 here
    assert _relres(A2, X, B) <= 1e-8
    assert np.linalg.norm(X - x_ref) <= 1e-6 * np.linalg.norm(x_ref)


def test_cg_with_the_factored_matrix_converges_at_once_and_host_equals_device():
    import torch

    A = M.grid_laplacian_3d(16, 3, 1e-2)
    c = CholeskyDecomposition(A.outer, A.inner, O.nested_dissection(A, 16))
    assert c.NumericFactorization(A.values, 0.5) == 0
    B = np.random.default_rng(3).standard_normal((A.n, 2))
    X, ok = c.ConjugateGradient(B, reg=0.5, relative_tolerance=1e-12)
    assert ok and c.IterationCount() <= 2
    shifted = M.CSRMatrix(n=A.n, outer=A.outer, inner=A.inner, values=A.values + 0.5 * (np.repeat(np.arange(A.n), np.diff(A.outer)) == A.inner))
    assert _relres(shifted, X, B) <= 1e-12
    Xd, okd = c.ConjugateGradient(torch.tensor(B, device="cuda"), reg=0.5, relative_tolerance=1e-12)
    # the column dot products accumulate atomically: equal to rounding, not bitwise
    assert okd and np.allclose(Xd.cpu().numpy(), X, rtol=1e-10, atol=1e-12 * np.abs(X).max())


def test_cg_alpha_beta_initial_guess_and_cap():
    A, A2, perm = _nearby_pair(14)
    c = CholeskyDecomposition(A.outer, A.inner, perm)
    assert c.NumericFactorization(A.values) == 0
    B = np.random.default_rng(4).standard_normal((A.n, 3))
    X, ok = c.ConjugateGradient(B, values=A2.values, relative_tolerance=1e-11, max_iter=300)
    assert ok
    # the solution as the initial guess: no steps
    X1, ok1 = c.ConjugateGradient(B, X=X.copy(), values=A2.values, relative_tolerance=1e-6, use_initial_guess=True)
    assert ok1 and c.IterationCount() == 0 and np.array_equal(X1, X)
    # X = alpha x + beta X
    X0 = np.random.default_rng(5).standard_normal(B.shape)
    X2, ok2 = c.ConjugateGradient(B, X=X0.copy(), values=A2.values, alpha=2.0, beta=0.5, relative_tolerance=1e-11, max_iter=300)
    assert ok2 and np.allclose(X2, 2.0 * X + 0.5 * X0, rtol=1e-6, atol=1e-6 * np.abs(X).max())
    # zero right-hand side and alpha = 0: X = beta X, converged
    X3, ok3 = c.ConjugateGradient(np.zeros_like(B), X=X0.copy(), values=A2.values, beta=3.0)
    assert ok3 and np.array_equal(X3, 3.0 * X0)
    X4, ok4 = c.ConjugateGradient(B, X=X0.copy(), alpha=0.0, beta=-1.0)
    assert ok4 and np.array_equal(X4, -X0)
    # the iteration cap: not converged, reported, X still written
    X5, ok5 = c.ConjugateGradient(B, values=A2.values, relative_tolerance=1e-14, max_iter=2)
    assert not ok5 and c.IterationCount() == 2 and np.all(np.isfinite(X5))


def test_cg_preconditioned_by_a_mixed_precision_factor():
    A = M.grid_laplacian_3d(18, 6, 1e-2)
    c = CholeskyDecomposition(A.outer, A.inner, O.nested_dissection(A, 16))
    c.SetPrecision("mixed")
    assert c.NumericFactorization(A.values) == 0
    B = np.random.default_rng(6).standard_normal((A.n, 2))
    X, ok = c.ConjugateGradient(B, relative_tolerance=1e-12, max_iter=50)
    assert ok and 1 <= c.IterationCount() <= 20
    assert _relres(A, X, B) <= 1e-9          # cond(A) < 1e5: |r| / |b| <= sqrt(cond) * 1e-12
