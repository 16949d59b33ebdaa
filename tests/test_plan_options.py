"""Device-plan options (trailing-update deferral, front relaxation, tensor-core tile width) and the
autotuner that picks them by timing.  On the CPU: every option set gives a plan that passes the
host-side plan check (every task in bounds, every update applied once) and the options change the
plan as intended.  On the GPU: factors under every option set match the oracle, and the autotuner
keeps the fastest candidate it timed."""
from __future__ import annotations

import itertools

import numpy as np
import pytest

import oracle
from tensors_b200 import matrices as M
from tensors_b200 import ordering as O
from tensors_b200.cholesky import CholeskyDecomposition, TBError


def _cases():
    A = M.grid_laplacian_3d(14, 0x5EED0041, 1e-2)
    B = M.vector_laplacian_3d(7, 0x5EED0042, 1e-2)
    return [(A, O.nested_dissection(A, 32)), (B, O.nested_dissection(B, 16))]


def test_every_option_set_passes_the_plan_check():
    for A, perm in _cases():
        c = CholeskyDecomposition(A.outer, A.inner, perm)
        c.SymbolicFactorization()
        sn = c.SN_Count()
        for d, r, w in itertools.product((1, 2, 3, 4), (0, 1, 2), (128, 256)):
            c.SetPlanOptions(d, r, w)
            assert c.PlanOptions() == (d, r, w)
            c.CheckPlan()
            assert c.SN_Count() == sn           # the symbolic analysis stands


def test_options_change_the_plan():
    A, perm = _cases()[0]
    c = CholeskyDecomposition(A.outer, A.inner, perm)
    c.SetPlanOptions(1, 1, 256)
    g1 = c.PlanStats()["gemm_tasks"]
    c.SetPlanOptions(3, 1, 256)
    g3 = c.PlanStats()["gemm_tasks"]
    assert g3 < g1                               # deferred updates: fewer, deeper tiles
    c.SetPlanOptions(3, 0, 256)
    f0 = c.PlanStats()["fronts"]
    c.SetPlanOptions(3, 2, 256)
    f2 = c.PlanStats()["fronts"]
    assert f2 < f0                               # looser relaxation merges more supernodes
    with pytest.raises(TBError):
        c.SetPlanOptions(5, 1, 256)


@pytest.mark.gpu
def test_factors_under_every_option_set_match_the_oracle():
    A, perm = _cases()[0]
    ref = oracle.OracleCholesky(A.n, A.outer, A.inner, perm)
    assert ref.factor(A.values, 0.0) == 0
    to, ro = ref.factor_values()
    B = np.random.default_rng(41).standard_normal((A.n, 3))
    Xo = ref.solve(B)
    for d, r in itertools.product((1, 2, 4), (0, 2)):
        c = CholeskyDecomposition(A.outer, A.inner, perm)
        c.SetPlanOptions(d, r, 256)
        assert c.NumericFactorization(A.values, 0.0) == 0
        tri, rec = c.FactorValues()
        scale = np.abs(to).max()
        assert max(np.abs(tri - to).max(), np.abs(rec - ro).max()) / scale < 1e-10, (d, r)
        assert np.abs(c.Solve(B) - Xo).max() / np.abs(Xo).max() < 1e-10, (d, r)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_plan_autotuner_keeps_the_fastest_and_a_valid_factor(precision):
    A = M.grid_laplacian_3d(24, 0x5EED0043, 1e-2)
    perm = O.graph_nested_dissection(A)
    c = CholeskyDecomposition(A.outer, A.inner, perm)
    c.SetPrecision(precision)
    c.SetRefinement(1e-10, 30)
    assert c.NumericFactorization(A.values, 0.0) == 0
    res = c.AutotunePlan()
    cands = [(d, r, w) for d in (2, 3, 4) for r in (0, 1, 2) for w in ((128, 256) if precision == "mixed" else (256,))]
    assert len(res["times_ms"]) == len(cands)
    assert res["choice"] == cands[int(np.argmin(res["times_ms"]))]
    assert c.PlanOptions() == res["choice"]
    print("plan autotuner", precision, "picked", res["choice"], "of", dict(zip(map(str, cands), np.round(res["times_ms"], 3))))
    # the handle is factored under the pick and solves to the target
    B = np.random.default_rng(43).standard_normal((A.n, 2))
    X = c.Solve(B)
    S = A.to_scipy()
    assert np.linalg.norm(B - S @ X) / np.linalg.norm(B) < 1e-10
