"""GPU parity on the benchmark configurations' own generators, against the
reference's own CPU code (oracle/_ref, the reference headers compiled in
place; the restatement when that library is absent).

The small cases of test_gpu_parity.py stop at 18^3 grids.  Here the fronts are
big enough for many 64-row panel steps and the deferred trailing updates:

* the 3D 7-point generator of the FP64 benchmark (lognormal(0,1) edge
  conductivities, shift 1e-6) on a 32^3 grid, under both nested dissections;
* the 3-dof 27-point vector-Laplacian generator of the mixed-precision
  benchmark (SPD 3x3 edge blocks G G^T + 0.1 I, shift 1e-2) on a 16^3 grid,
  in FP64 and in mixed precision with FP64 refinement;
* the Delaunay generator of the batched benchmark: the worst-conditioned
  systems of its first 100 meshes.

Checked against the reference: factor entries (max-norm, relative to the
largest entry), the forward difference of the solutions, and both relative
residuals ||B - A X|| / ||B||.  Tolerances are written beside each check.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

import oracle
from tensors_b200 import matrices as M
from tensors_b200 import ordering as O
from tensors_b200.cholesky import CholeskyDecomposition

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


def reference(A, perm):
    """The reference's own factorization (Maximal supernodes), or the restatement without it."""
    if oracle.ref_available():
        ref = oracle.RefCholesky(A.n, A.outer, A.inner, perm, "maximal", threads=THREADS, blas_threads=1)
        ref.symbolic()
        return ref
    return oracle.OracleCholesky(A.n, A.outer, A.inner, perm, "maximal")


def ref_solve(ref, B):
    return ref.solve(B, parallel=False) if isinstance(ref, oracle.RefCholesky) else ref.solve(B)


def relres(A, X, B, reg=0.0):
    S = A.to_scipy()
    R = B - S @ X - reg * X
    return float(np.linalg.norm(R) / np.linalg.norm(B))


def factor_diff(chol, ref):
    tri, rec = chol.FactorValues()
    to, ro = ref.factor_values()
    assert tri.shape == to.shape and rec.shape == ro.shape
    scale = np.abs(to).max()
    d = np.abs(tri - to).max() / scale
    if len(ro):
        d = max(d, np.abs(rec - ro).max() / scale)
    return float(d)


def fwd_diff(X, Xo):
    return float(np.linalg.norm(X - Xo) / np.linalg.norm(Xo))


@pytest.mark.parametrize("ordering", ["geometric", "graph"])
def test_fp64_benchmark_generator_32cubed_matches_reference(ordering):
    A = M.grid_laplacian_3d(32, 0x5EED0002, 1e-6)
    perm = O.nested_dissection(A) if ordering == "geometric" else O.graph_nested_dissection(A)
    chol = CholeskyDecomposition(A.outer, A.inner, perm)
    chol.CheckPlan()
    ref = reference(A, perm)
    assert chol.NumericFactorization(A.values, 0.0) == 0
    assert ref.factor(A.values, 0.0) == 0
    # many panel steps: the largest front spans several 64-row panels
    assert chol.PlanStats()["levels"] > 4
    # factor entries: the same FP64 arithmetic in another order
    assert factor_diff(chol, ref) < 1e-10
    B = np.random.default_rng(0x5EED0002 + 1).standard_normal((A.n, 16))
    X = chol.Solve(B)
    Xo = ref_solve(ref, B)
    # kappa(A) <= 2 max(diag) / 1e-6 (Gershgorin over the shift, the smallest
    # eigenvalue: constants span the Laplacian's null space), ~1e9 here; two
    # backward-stable solves differ by at most ~kappa * u
    kappa = 2.0 * A.to_scipy().diagonal().max() / 1e-6
    assert fwd_diff(X, Xo) < 10 * kappa * 2.2e-16
    assert relres(A, X, B) < 1e-10
    assert relres(A, Xo, B) < 1e-10
    assert abs(chol.LogDeterminant() - ref.log_det()) <= 1e-10 * abs(ref.log_det())


def test_vector_laplacian_generator_16cubed_fp64_and_mixed_match_reference():
    A = M.vector_laplacian_3d(16, 0x5EED0003, 1e-2)
    perm = O.nested_dissection(A)
    ref = reference(A, perm)
    assert ref.factor(A.values, 0.0) == 0
    B = np.random.default_rng(0x5EED0003 + 1).standard_normal((A.n, 8))
    Xo = ref_solve(ref, B)
    rr_ref = relres(A, Xo, B)
    assert rr_ref < 1e-12

    chol = CholeskyDecomposition(A.outer, A.inner, perm)
    chol.CheckPlan()
    assert chol.NumericFactorization(A.values, 0.0) == 0
    assert factor_diff(chol, ref) < 1e-10
    X = chol.Solve(B)
    assert fwd_diff(X, Xo) < 1e-11
    assert relres(A, X, B) < 1e-12

    # mixed precision: FP32 factor with 3xTF32 updates, refined in FP64 to 1e-10 and to 1e-12
    mixed = CholeskyDecomposition(A.outer, A.inner, perm)
    mixed.SetPrecision("mixed")
    for tol in (1e-10, 1e-12):
        mixed.SetRefinement(tol, 30)
        assert mixed.NumericFactorization(A.values, 0.0) == 0
        Xm = mixed.Solve(B)
        assert mixed.PrecisionInUse()[0] == "mixed"
        rr = relres(A, Xm, B)
        assert rr <= tol, (tol, rr)
        # forward difference against the reference's FP64 solution: kappa ~1e3 here
        # (stiffness eigenvalues up to ~1e1 over the 1e-2 shift), so ~kappa x the residual
        assert fwd_diff(Xm, Xo) < 1e4 * tol
    # the FP32 factor is a backward-stable factor of A at FP32 precision; its
    # entries' forward error against the FP64 factor grows like kappa(A) (~1e3
    # here) x the FP32 unit roundoff 2^-24, so the bound is 1e4 x 2^-24
    assert factor_diff(mixed, ref) < 1e4 * 2.0 ** -24


def _c4_worst(count=100, worst=25):
    """The `worst` systems of the batch generator's first `count` meshes by max(diag) / min(diag)."""
    ms = np.random.default_rng(0x5EED0004).integers(500, 20001, size=count)
    out = []
    for s in range(count):
        A = M.delaunay_laplacian(int(ms[s]), 0x5EED0004 + s, 1e-3)
        d = A.to_scipy().diagonal()
        out.append((float(d.max() / d.min()), s, A))
    out.sort(key=lambda e: -e[0])
    return out[:worst]


def backward_error(A, X, B):
    """Normwise backward error ||B - A X||_inf / (||A||_inf ||X||_inf + ||B||_inf)."""
    S = A.to_scipy()
    R = B - S @ X
    norm_a = float(abs(S).sum(axis=1).max())
    return float(np.abs(R).max() / (norm_a * np.abs(X).max() + np.abs(B).max()))


def test_batch_generator_worst_systems_fp64_residual_matches_reference():
    """On the most ill-conditioned Delaunay systems (cotangent weights of near-flat hull triangles
    against a tiny lumped mass) the GPU's FP64 factor + solve is backward stable like the
    reference's own FP64 code: normwise backward error below 1e-15 (~4.5 x 2^-53) and within 8x of
    the reference's.  The relative residual ||b - A x|| / ||b|| is kappa(A) x the backward error
    and varies with the summation order alone: on system 53 (n = 13573) four FP64 multifrontal
    factorizations that differ only in the order of their roundings (triangular solves by
    substitution or by explicit 64 x 64 inverses, the restatement, the reference) give
    2.1e-9 to 6.8e-9, all at backward error 0.5e-16 to 1.7e-16.  So the residual is held to 8x
    the reference's, or below 1e-14."""
    rows = []
    for proxy, s, A in _c4_worst():
        perm = O.nested_dissection(A)
        ref = reference(A, perm)
        assert ref.factor(A.values, 0.0) == 0
        b = np.random.default_rng(0x5EED0004 + 1 + s).standard_normal((A.n, 1))
        x_ref = ref_solve(ref, b)
        chol = CholeskyDecomposition(A.outer, A.inner, perm)
        assert chol.NumericFactorization(A.values, 0.0) == 0
        x = chol.Solve(b)
        rows.append((s, A.n, proxy, relres(A, x, b), relres(A, x_ref, b),
                     backward_error(A, x, b), backward_error(A, x_ref, b)))
    bad = [r for r in rows if not (r[3] <= max(8.0 * r[4], 1e-14) and r[5] <= 1e-15 and r[5] <= max(8.0 * r[6], 1e-16))]
    assert not bad, ("system, n, diag ratio, GPU relres, reference relres, GPU backward error, "
                     "reference backward error: " + repr(bad))
