"""Mixed precision: FP32 factor with 3xTF32 Schur updates, FP64 refinement.

The refined solution must reach the requested relative residual
max_c |b_c - (A + reg I) x_c| / |b_c| and agree with the FP64 path to the
accuracy the conditioning allows; the FP32 factor itself must be a backward-stable
factorization at single precision (|P A P^T - U^T U| / |A| < 1e-6).
"""
from __future__ import annotations

import numpy as np
import pytest

from tensors_b200 import matrices as M
from tensors_b200 import ordering as O
from tensors_b200.cholesky import CholeskyDecomposition

pytestmark = pytest.mark.gpu


def _cases():
    out = []
    A = M.grid_laplacian_2d(64, 0.0)
    out.append(("c1-grid2d-64", A, O.nested_dissection(A), 1e-2))
    A = M.grid_laplacian_3d(16, 3, 1e-2)
    out.append(("grid3d-16", A, O.nested_dissection(A), 0.0))
    A = M.vector_laplacian_3d(7, 4, 1e-2)
    out.append(("vector3d-7", A, O.nested_dissection(A), 0.0))
    A = M.delaunay_laplacian(4000, 5)
    out.append(("delaunay-4000", A, O.nested_dissection(A), 0.0))
    A = M.grid_laplacian_3d(26, 6, 1e-2)                 # top fronts with several panels
    out.append(("grid3d-26", A, O.nested_dissection(A), 0.0))
    return out


CASES = _cases()


def factor_backward_error(chol, A, reg):
    import scipy.sparse as sp

    p = chol.GetPermutation()
    S = (A.to_scipy() + reg * sp.identity(A.n)).tocsr()[p][:, p]
    U = chol.GetU()
    E = (U.T @ U - S)
    return float(sp.linalg.norm(E) / sp.linalg.norm(S))


def backward_error(A, X, B, reg):
    S = A.to_scipy()
    R = B - S @ X - reg * X
    nA = abs(S).sum(axis=1).max() + reg
    return float(np.linalg.norm(R, np.inf) / (nA * np.linalg.norm(X, np.inf) + np.linalg.norm(B, np.inf)))


def relres(A, X, B, reg):
    R = B - A.to_scipy() @ X - reg * X
    return float(np.max(np.linalg.norm(R, axis=0) / np.linalg.norm(B, axis=0)))


@pytest.mark.parametrize("name,A,perm,reg", CASES, ids=[c[0] for c in CASES])
def test_mixed_precision_refines_to_tolerance(name, A, perm, reg):
    B = np.random.default_rng(A.n).standard_normal((A.n, 4))
    ref = CholeskyDecomposition(A.outer, A.inner, perm)
    assert ref.NumericFactorization(A.values, reg) == 0
    X64 = ref.Solve(B)
    # what a backward-stable FP64 solve attains on this matrix (for kappa ~1e9
    # a relative residual of 1e-12 is out of reach of any FP64 solver)
    target = max(1e-12, 4.0 * relres(A, X64, B, reg))

    mix = CholeskyDecomposition(A.outer, A.inner, perm)
    mix.SetPrecision("mixed")
    mix.SetRefinement(target, 60)
    assert mix.NumericFactorization(A.values, reg) == 0
    X = mix.Solve(B)
    it, rr = mix.RefinementInfo()
    assert rr <= target, (it, rr, target)
    assert relres(A, X, B, reg) <= 2 * target
    assert it >= 1                                        # an FP32 factor alone does not reach the target
    # forward error: both solutions are within kappa * residual of the exact one
    assert backward_error(A, X, B, reg) < 1e-14

    # the FP32 factor is a backward-stable factorization at single precision:
    # |P (A + reg I) P^T - U^T U|_F / |A + reg I|_F at FP32 rounding level
    assert factor_backward_error(mix, A, reg) < 1e-6
    assert factor_backward_error(ref, A, reg) < 1e-14


def test_mixed_half_solves_and_precision_switch():
    A = M.grid_laplacian_3d(12, 9, 1e-2)
    perm = O.nested_dissection(A, 16)
    c = CholeskyDecomposition(A.outer, A.inner, perm)
    B = np.random.default_rng(1).standard_normal((A.n, 2))
    assert c.NumericFactorization(A.values) == 0
    y64 = c.UpperSolve(B)
    x64 = c.Solve(B)
    c.SetPrecision("mixed")
    assert not c.NumericallyFactorizedQ()
    assert c.NumericFactorization(A.values) == 0
    y32 = c.UpperSolve(B)                                 # one application of the FP32 factor, no refinement
    assert np.abs(y32 - y64).max() / np.abs(y64).max() < 1e-5
    x32 = c.Solve(B)
    assert np.abs(x32 - x64).max() / np.abs(x64).max() < 1e-10
    c.SetPrecision("fp64")
    assert c.NumericFactorization(A.values) == 0
    x = c.Solve(B)
    assert np.abs(x - x64).max() / np.abs(x64).max() < 1e-13


@pytest.mark.parametrize("schedule", ["task_graph", "task_graph_all"])
def test_mixed_task_graph_matches_levels_bitwise(schedule):
    A = M.grid_laplacian_3d(24, 13, 1e-2)
    perm = O.nested_dissection(A, 64)
    a = CholeskyDecomposition(A.outer, A.inner, perm)
    b = CholeskyDecomposition(A.outer, A.inner, perm)
    for h in (a, b):
        h.SetPrecision("mixed")
    a.SetSchedule(schedule)
    b.SetSchedule("levels")
    assert a.NumericFactorization(A.values) == 0
    assert b.NumericFactorization(A.values) == 0
    ta, ra = a.FactorValues()
    tb_, rb = b.FactorValues()
    assert np.array_equal(ta, tb_) and np.array_equal(ra, rb)


def test_mixed_factor_stays_finite_when_pivots_are_raised():
    # A Delaunay system of the batched workload (cotangent Laplacian of 13,580
    # random points + 1e-3 lumped mass, kappa ~1e10) on which FP32 rounding
    # wipes out several pivots.  Raised pivots must not let the rows below them
    # grow until FP32 overflows (which left NaN in the factor before the growth
    # bound); the refined solve then reaches what FP64 reaches.
    seed = 0x5EED0004
    m = np.random.default_rng(seed).integers(500, 20001, size=25)[24]
    A = M.delaunay_laplacian(int(m), seed + 24, 1e-3)
    perm = O.nested_dissection(A)
    B = np.random.default_rng(7).standard_normal((A.n, 2))
    ref = CholeskyDecomposition(A.outer, A.inner, perm)
    assert ref.NumericFactorization(A.values, 0.0) == 0
    target = max(1e-10, 4.0 * relres(A, ref.Solve(B), B, 0.0))

    mix = CholeskyDecomposition(A.outer, A.inner, perm)
    mix.SetPrecision("mixed")
    mix.SetRefinement(target, 100)
    assert mix.NumericFactorization(A.values, 0.0) == 0
    tri, rec = mix.FactorValues()
    assert np.isfinite(tri).all() and np.isfinite(rec).all(), mix.PerturbedPivots()
    X = mix.Solve(B)
    it, rr = mix.RefinementInfo()
    assert np.isfinite(X).all() and rr <= target, (it, rr, target, mix.PerturbedPivots())
    assert relres(A, X, B, 0.0) <= 2 * target
    # whether the FP32 factor sufficed or the solve fell back to an FP64 factor,
    # the handle says which, and a new precision setting clears the fallback
    used, fell_back = mix.PrecisionInUse()
    assert (used, fell_back) in (("mixed", False), ("fp64", True))
    if fell_back:
        tri, rec = mix.FactorValues()
        assert np.isfinite(tri).all() and np.isfinite(rec).all()
    mix.SetPrecision("mixed")
    assert mix.PrecisionInUse() == ("mixed", False)
