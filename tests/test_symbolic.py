"""Host-side symbolic analysis and device plan, through the C-ABI (no GPU).

The product's symbolic analysis must reproduce the reference's integer
structure exactly; it is compared with the oracle (itself pinned to the
reference) on grids, random permutations, meshes and forests, for all three
supernode strategies.  Every device plan is bounds-checked on the host.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from tensors_b200 import matrices as M
from tensors_b200 import ordering as O
from tensors_b200.cholesky import CholeskyDecomposition, TBError

STRATS = {"maximal": 0, "fundamental": 1, "amalgamated": 2}


def _cases():
    out = []
    for g in (1, 2, 7, 30):
        A = M.grid_laplacian_2d(g, 1.0)
        out.append((f"grid2d-{g}", A, O.nested_dissection(A, 8) if g > 1 else None))
        if g > 1:
            out.append((f"grid2d-{g}-rand", A, np.random.default_rng(g).permutation(A.n).astype(np.int32)))
    A = M.grid_laplacian_3d(14, 3)
    out.append(("grid3d-14", A, O.nested_dissection(A, 32)))
    A = M.vector_laplacian_3d(5, 4)
    out.append(("vector3d-5", A, O.nested_dissection(A, 8)))
    A = M.delaunay_laplacian(2500, 5)
    out.append(("delaunay-2500", A, O.nested_dissection(A, 16)))
    out.append(("delaunay-2500-rand", A, np.random.default_rng(9).permutation(A.n).astype(np.int32)))
    # the ordering from the pattern alone (other front shapes than the geometric one)
    out.append(("delaunay-2500-graph", A, O.graph_nested_dissection(A, 16)))
    A = M.grid_laplacian_3d(14, 3)
    out.append(("grid3d-14-graph", A, O.graph_nested_dissection(A, 32)))
    A = M.vector_laplacian_3d(5, 4)
    out.append(("vector3d-5-graph", A, O.graph_nested_dissection(A, 8)))
    return out


CASES = _cases()


@pytest.mark.parametrize("strategy", list(STRATS))
@pytest.mark.parametrize("name,A,perm", CASES, ids=[c[0] for c in CASES])
def test_symbolic_matches_oracle(name, A, perm, strategy):
    o = oracle.OracleCholesky(A.n, A.outer, A.inner, perm, strategy)
    c = CholeskyDecomposition(A.outer, A.inner, perm)
    c.SetSupernodeStrategy(STRATS[strategy])
    for key in oracle.ARRAYS:
        assert np.array_equal(c.SymbolicArray(key), o.array(key)), key
    assert c.SN_Count() == o.sn_count()
    c.CheckPlan()
    st = c.PlanStats()
    assert 1 <= st["fronts"] <= st["supernodes"] == o.sn_count()
    f, nnz_u = c.FlopCount()
    n0 = np.diff(o.array("SN_rp")).astype(float)
    n1 = np.diff(o.array("SN_outer")).astype(float)
    assert np.isclose(f, (n0 ** 3 / 3 + n0 ** 2 * n1 + n0 * n1 ** 2).sum())
    assert np.isclose(nnz_u, (n0 * (n0 + 1) / 2 + n0 * n1).sum())


def test_unsorted_rows_accepted_with_permutation():
    A = M.grid_laplacian_2d(9, 1.0)
    perm = O.nested_dissection(A, 8)
    inner = A.inner.copy()
    for i in range(A.n):            # reverse every row
        inner[A.outer[i]:A.outer[i + 1]] = inner[A.outer[i]:A.outer[i + 1]][::-1]
    c1 = CholeskyDecomposition(A.outer, A.inner, perm)
    c2 = CholeskyDecomposition(A.outer, inner, perm)
    for key in ("SN_rp", "SN_outer", "SN_inner", "perm", "inner"):
        assert np.array_equal(c1.SymbolicArray(key), c2.SymbolicArray(key))
    # the value permutation follows the moved entries
    v1, v2 = c1.GetValuePermutation(), c2.GetValuePermutation()
    rows = np.repeat(np.arange(A.n), np.diff(A.outer))
    rev = np.empty_like(inner)
    for i in range(A.n):
        b, e = A.outer[i], A.outer[i + 1]
        rev[b:e] = np.arange(e - 1, b - 1, -1)
    assert np.array_equal(rev[v2], v1)


@pytest.mark.parametrize("bad", ["not_permutation", "missing_diagonal", "unsorted_without_perm", "out_of_range"])
def test_invalid_inputs_are_rejected(bad):
    A = M.grid_laplacian_2d(6, 1.0)
    outer, inner, perm = A.outer.copy(), A.inner.copy(), O.nested_dissection(A, 4)
    if bad == "not_permutation":
        perm = perm.copy()
        perm[0] = perm[1]
    elif bad == "missing_diagonal":
        # drop the diagonal entry of row 3
        rows = np.repeat(np.arange(A.n), np.diff(outer))
        keep = ~((rows == 3) & (inner == 3))
        inner = inner[keep]
        outer = np.concatenate([[0], np.cumsum(np.bincount(rows[keep], minlength=A.n))]).astype(np.int64)
    elif bad == "unsorted_without_perm":
        inner[outer[2]:outer[3]] = inner[outer[2]:outer[3]][::-1]
        perm = None
    elif bad == "out_of_range":
        inner[5] = A.n + 3
    c = CholeskyDecomposition(outer, inner, perm)
    with pytest.raises(TBError):
        c.SymbolicFactorization()


def test_setters_invalidate_symbolic():
    A = M.grid_laplacian_2d(16, 1.0)
    c = CholeskyDecomposition(A.outer, A.inner, O.nested_dissection(A, 8))
    n_max = c.SN_Count()
    c.SetSupernodeStrategy(2)
    c.SetAmalgamationThreshold(8)
    o = oracle.OracleCholesky(A.n, A.outer, A.inner, O.nested_dissection(A, 8), "amalgamated", 8)
    assert c.SN_Count() == o.sn_count() != n_max


def test_relaxed_fronts_cover_supernodes_and_reduce_levels():
    A = M.grid_laplacian_3d(24, 1)
    c = CholeskyDecomposition(A.outer, A.inner, O.nested_dissection(A))
    st = c.PlanStats()
    assert st["fronts"] < st["supernodes"]
    assert st["levels"] < 40
    c.CheckPlan()


@pytest.mark.parametrize("grid,leaf", [(12, 8), (20, 32), (16, 64)])
def test_solve_task_graph_plan_is_deadlock_free(grid, leaf):
    # host side of the persistent solve: for every solve schedule the plan
    # check verifies the task lists (every update of a panel comes before the
    # panel's first forward task; every task of a target panel before the back
    # task that reads it) and the flop invariant of the deferred updates
    A = M.grid_laplacian_3d(grid, 17, 1e-3)
    c = CholeskyDecomposition(A.outer, A.inner, O.nested_dissection(A, leaf))
    c.SymbolicFactorization()
    c.CheckPlan()
    assert c.PlanStats()["solve_graph_tasks"] == 0            # level launches by default
    tasks = {}
    for sched in ("task_graph_all", "task_graph", "levels"):
        c.SetSolveSchedule(sched)
        c.CheckPlan()
        tasks[sched] = c.PlanStats()["solve_graph_tasks"]
    assert tasks["levels"] == 0
    assert tasks["task_graph_all"] > 0 and tasks["task_graph_all"] >= tasks["task_graph"]


def test_u_nonzero_count_matches_the_flop_count_structure():
    for A in (M.grid_laplacian_2d(30, 1.0), M.delaunay_laplacian(2500, 5)):
        c = CholeskyDecomposition(A.outer, A.inner, O.nested_dissection(A, 16))
        c.SymbolicFactorization()
        rp, so = c.SymbolicArray("SN_rp"), c.SymbolicArray("SN_outer")
        n0, n1 = np.diff(rp), np.diff(so)
        assert c.UNonzeroCount() == int(np.sum(n0 * (n0 + 1) // 2 + n0 * n1))
        assert c.UNonzeroCount() == int(c.FlopCount()[1])


def test_settings_getters_follow_the_setters():
    from tensors_b200.cholesky import FactorizationMethod, SupernodeStrategy

    A = M.grid_laplacian_2d(8, 1.0)
    c = CholeskyDecomposition(A.outer, A.inner, thread_count=2)
    assert (c.GetSupernodeStrategy(), c.AmalgamationThreshold(), c.GetFactorizationMethod(), c.ThreadCount()) == \
        (SupernodeStrategy.Maximal, 4, FactorizationMethod.Multifrontal, 2)
    c.SetSupernodeStrategy(SupernodeStrategy.Amalgamated)
    c.SetAmalgamationThreshold(7)
    c.SetFactorizationMethod(FactorizationMethod.LeftLooking)
    assert (c.GetSupernodeStrategy(), c.AmalgamationThreshold(), c.GetFactorizationMethod()) == \
        (SupernodeStrategy.Amalgamated, 7, FactorizationMethod.LeftLooking)


@pytest.mark.parametrize("order", ["geometric", "pattern"])
def test_analysis_is_the_same_on_any_number_of_threads(order):
    # the elimination tree runs in row chunks (one per thread, from 2 x 65,536 rows on) merged
    # by a serial pass, and the supernode starts are decided row-parallel: the symbolic arrays
    # are those of one thread, for an ordering that is already postordered (the geometric
    # dissection) and one that is not (the dissection from the pattern alone)
    A = M.grid_laplacian_2d(730, 1.0)         # 532,900 rows: up to 8 chunks
    perm = O.nested_dissection(A, 64) if order == "geometric" else O.graph_nested_dissection(A, 64)
    got = {}
    for threads in (1, 2, 3, 8):
        c = CholeskyDecomposition(A.outer, A.inner, perm, thread_count=threads)
        c.SymbolicFactorization()
        got[threads] = (c.EliminationTreeParents(), c.GetPermutation(), c.GetValuePermutation(), c.SN_RowPointers(),
                        c.SN_Outer(), c.SN_Inner(), c.AssemblyTreeParents())
    for threads in (2, 3, 8):
        for a, b in zip(got[1], got[threads]):
            assert np.array_equal(a, b), threads
