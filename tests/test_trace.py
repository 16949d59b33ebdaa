"""Phase ranges: the path's phases appear as ranges named with the reference's
TOOLS_PTIMER tags (Symbolic.hpp:7, EliminationTree.hpp:11, CholeskyDecomposition.hpp:391/433,
Symbolic.hpp:266, AssemblyTree.hpp:14, Numeric.hpp:34/167/258, Solve.hpp:42/351/392)."""
from __future__ import annotations

import numpy as np
import pytest

from tensors_b200 import matrices as M
from tensors_b200 import ordering as O
from tensors_b200 import trace
from tensors_b200.cholesky import CholeskyDecomposition

P = "Sparse::CholeskyDecomposition::"


def test_symbolic_phases_are_ranges():
    A = M.grid_laplacian_2d(12, 1.0)
    perm = np.random.default_rng(5).permutation(A.n).astype(np.int32)   # not postordered
    with trace.recording() as got:
        c = CholeskyDecomposition(A.outer, A.inner, perm)
        c.SymbolicFactorization()
    for tag in ("SymbolicFactorization", "Init", "EliminationTree", "PostOrdering", "FindMaximalSupernodes",
                "CreateAssemblyTree"):
        assert P + tag in got, tag
    assert got.index(P + "SymbolicFactorization") < got.index(P + "CreateAssemblyTree")
    # nothing is recorded once recording stops
    c2 = CholeskyDecomposition(A.outer, A.inner, perm)
    c2.SetSupernodeStrategy(1)
    c2.SymbolicFactorization()
    assert trace.names() == []


def test_phase_times_nest():
    # every closed range has a host duration, and the enclosing SymbolicFactorization range
    # lasts at least as long as the steps inside it
    A = M.grid_laplacian_2d(40, 1.0)
    trace.record(True)
    try:
        c = CholeskyDecomposition(A.outer, A.inner, O.nested_dissection(A, 8))
        c.SymbolicFactorization()
        got = trace.times()
    finally:
        trace.record(False)
    d = dict(got)
    assert all(t >= 0.0 for _, t in got)
    inner = sum(d[P + tag] for tag in ("Init", "EliminationTree", "PostOrdering", "FindMaximalSupernodes",
                                       "CreateAssemblyTree") if P + tag in d)
    assert d[P + "SymbolicFactorization"] >= inner
    assert trace.times() == []


def test_strategy_names_its_supernode_range():
    A = M.grid_laplacian_2d(10, 1.0)
    for strategy, tag in ((1, "FindFundamentalSupernodes"), (2, "FindAmalgamatedSupernodes")):
        with trace.recording() as got:
            c = CholeskyDecomposition(A.outer, A.inner, O.nested_dissection(A, 8))
            c.SetSupernodeStrategy(strategy)
            c.SymbolicFactorization()
        assert P + tag in got


@pytest.mark.gpu
def test_numeric_and_solve_phases_are_ranges():
    A = M.grid_laplacian_2d(16, 1.0)
    c = CholeskyDecomposition(A.outer, A.inner, O.nested_dissection(A, 8))
    c.SymbolicFactorization()
    with trace.recording() as got:
        assert c.NumericFactorization(A.values, 0.0) == 0
        c.Solve(np.ones(A.n))
    for tag in ("NumericFactorization_Multifrontal", "ClearFactors", "ReadNonzeroValues", "Solve", "SN_LowerSolve",
                "SN_UpperSolve"):
        assert P + tag in got, tag
