"""The super-panel solve of large fronts: fronts with at least 256 pivot rows step through
their rows 512 at a time with the inverse of each 512 x 512 diagonal block (formed after the
factorization from the 64-row panel inverses).  On the CPU: the plan has super-panels for such
fronts, and the checked launch lists cover every task once.  On the GPU: solves match the oracle
in FP64 and reach the refinement target in mixed precision, for RHS counts below, at and above one
sweep chunk, and agree with the panel-step sweeps (the no-allocation solve keeps those)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from tensors_b200 import _lib
from tensors_b200 import matrices as M
from tensors_b200 import ordering as O
from tensors_b200.cholesky import CholeskyDecomposition


def _big():
    A = M.grid_laplacian_3d(40, 0x5EED0061, 1e-3)          # top separator 40 x 40 = 1600 rows
    return A, O.nested_dissection(A)


def test_large_fronts_get_super_panels():
    A, perm = _big()
    c = CholeskyDecomposition(A.outer, A.inner, perm)
    c.CheckPlan()
    st = c.PlanStats()
    assert st["super_panels"] >= 4
    assert st["lower_launches_super"] < st["lower_launches"]
    small = M.grid_laplacian_3d(10, 1, 1e-2)
    c2 = CholeskyDecomposition(small.outer, small.inner, O.nested_dissection(small))
    assert c2.PlanStats()["super_panels"] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("k", [1, 8, 17, 70])
def test_super_panel_solves_match_the_oracle(k):
    A, perm = _big()
    c = CholeskyDecomposition(A.outer, A.inner, perm)
    assert c.NumericFactorization(A.values, 0.0) == 0
    ref = oracle.OracleCholesky(A.n, A.outer, A.inner, perm)
    assert ref.factor(A.values, 0.0) == 0
    B = np.random.default_rng(61 + k).standard_normal((A.n, k))
    X = c.Solve(B)
    Xo = ref.solve(B)
    assert np.abs(X - Xo).max() / np.abs(Xo).max() < 1e-9
    S = A.to_scipy()
    assert np.linalg.norm(B - S @ X) / np.linalg.norm(B) < 1e-11
    # the half solves keep the panel steps' meaning
    Xu = c.UpperSolve(B)
    assert np.abs(Xu - ref.solve(B, which="upper")).max() / np.abs(Xu).max() < 1e-9


@pytest.mark.gpu
def test_super_panel_sweeps_agree_with_panel_step_sweeps():
    import torch

    A, perm = _big()
    c = CholeskyDecomposition(A.outer, A.inner, perm)
    assert c.NumericFactorization(A.values, 0.0) == 0
    k = 6
    B = torch.tensor(np.random.default_rng(62).standard_normal((A.n, k)), device="cuda")
    X1 = torch.zeros_like(B)
    X2 = torch.zeros_like(B)
    lib = _lib.lib()
    assert lib.tb_chol_solve_device(c.handle, 1.0, B.data_ptr(), k, 0.0, X1.data_ptr(), k, k) == 0
    assert lib.tb_chol_solve_device_noalloc(c.handle, 1.0, B.data_ptr(), k, 0.0, X2.data_ptr(), k, k) == 0
    torch.cuda.synchronize()
    assert float((X1 - X2).abs().max() / X2.abs().max()) < 1e-12


@pytest.mark.gpu
def test_super_panel_solves_in_mixed_precision():
    A = M.vector_laplacian_3d(20, 0x5EED0063, 1e-2)         # top separator 20 x 20 x 3 = 1200 rows
    c = CholeskyDecomposition(A.outer, A.inner, O.nested_dissection(A))
    assert c.PlanStats()["super_panels"] >= 3
    c.SetPrecision("mixed")
    c.SetRefinement(1e-11, 30)
    assert c.NumericFactorization(A.values, 0.0) == 0
    B = np.random.default_rng(63).standard_normal((A.n, 8))
    X = c.Solve(B)
    assert c.PrecisionInUse() == ("mixed", False)
    S = A.to_scipy()
    assert np.linalg.norm(B - S @ X) / np.linalg.norm(B) <= 1e-11
