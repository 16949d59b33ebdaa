"""GPU parity: the CUDA factorization and solves against the CPU oracle.

The oracle (oracle/oracle.cpp) restates the reference's multifrontal
algorithm and is itself pinned to the reference's own code (see
test_oracle_reference.py).  Integer structure must match exactly; factor
entries must agree to FP64 rounding (relative max-norm tolerance 1e-10: the
same FP64 arithmetic in a different order).  Solutions of a system with
condition number kappa can differ by ~kappa * 1e-16 between two backward
stable solvers, so solutions are compared at 1e-10 for the well-conditioned
cases and at a per-case tolerance for the ill-conditioned ones, and both
solvers' normwise backward errors ||b - A x|| / (||A|| ||x|| + ||b||) must be
below 1e-14.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import oracle
from tensors_b200 import matrices as M
from tensors_b200 import ordering as O
from tensors_b200._lib import lib
from tensors_b200.cholesky import CholeskyDecomposition, TBError

pytestmark = pytest.mark.gpu

TOL = 1e-10


def rel_err(x, y):
    scale = max(np.abs(y).max(initial=0.0), 1e-300)
    return float(np.abs(np.asarray(x) - np.asarray(y)).max(initial=0.0) / scale)


def _cases():
    # (name, matrix, permutation, diagonal shift, solution tolerance)
    out = []
    for g in (3, 8, 33):
        A = M.grid_laplacian_2d(g, 0.0)
        out.append((f"grid2d-{g}-nd", A, O.nested_dissection(A, 8), 1e-2, TOL))
        out.append((f"grid2d-{g}-rand", A, np.random.default_rng(g).permutation(A.n).astype(np.int32), 1e-2, TOL))
    A = M.grid_laplacian_3d(12, 7, 1e-6)              # kappa ~ 1e7
    out.append(("grid3d-12", A, O.nested_dissection(A, 16), 0.0, 1e-8))
    A = M.grid_laplacian_3d(18, 5, 1e-2)              # fronts with several panels and > 256 rest columns
    out.append(("grid3d-18", A, O.nested_dissection(A, 64), 0.0, TOL))
    out.append(("grid3d-18-graph", A, O.graph_nested_dissection(A, 64), 0.0, TOL))   # ordering from the pattern
    A = M.vector_laplacian_3d(6, 8)
    out.append(("vector3d-6", A, O.nested_dissection(A, 16), 1e-2, TOL))
    A = M.delaunay_laplacian(3000, 9)                 # shift 1e-3 * lumped mass: kappa ~ 1e9
    out.append(("delaunay-3000", A, O.nested_dissection(A, 16), 0.0, 1e-6))
    A = M.grid_laplacian_2d(20, 1.0)
    out.append(("grid2d-20-identity-perm", A, None, 0.0, TOL))
    A = M.grid_laplacian_2d(64, 0.0)                  # the reference's CPU case: 64^2 grid, shift 1e-2
    out.append(("c1-grid2d-64", A, O.nested_dissection(A), 1e-2, TOL))
    return out


CASES = _cases()


def backward_error(A, X, B, reg=0.0):
    S = A.to_scipy()
    R = B - S @ X - reg * X
    nA = abs(S).sum(axis=1).max() + reg
    return float(np.linalg.norm(R, np.inf) / (nA * np.linalg.norm(X, np.inf) + np.linalg.norm(B, np.inf)))


@pytest.mark.parametrize("strategy", [0, 1, 2])
@pytest.mark.parametrize("name,A,perm,reg,sol_tol", CASES, ids=[c[0] for c in CASES])
def test_factor_and_solve_match_oracle(name, A, perm, reg, sol_tol, strategy):
    chol = CholeskyDecomposition(A.outer, A.inner, perm)
    chol.SetSupernodeStrategy(strategy)
    ref = oracle.OracleCholesky(A.n, A.outer, A.inner, perm, ["maximal", "fundamental", "amalgamated"][strategy])
    chol.CheckPlan()
    assert chol.NumericFactorization(A.values, reg) == 0
    assert ref.factor(A.values, reg) == 0
    assert chol.NumericallyFactorizedQ() and chol.NumericallyGoodQ()

    for key in oracle.ARRAYS:
        assert np.array_equal(chol.SymbolicArray(key), ref.array(key)), key

    tri, rec = chol.FactorValues()
    to, ro = ref.factor_values()
    assert tri.shape == to.shape and rec.shape == ro.shape
    scale = np.abs(to).max()
    assert np.abs(tri - to).max() / scale < TOL
    if len(ro):
        assert np.abs(rec - ro).max() / scale < TOL
    # the strictly lower part of every U0 square stays exactly zero
    rp, tp = chol.SN_RowPointers(), chol.SN_TrianglePointers()
    for s in range(len(rp) - 1):
        n0 = rp[s + 1] - rp[s]
        U0 = tri[tp[s]:tp[s] + n0 * n0].reshape(n0, n0)
        assert not np.tril(U0, -1).any()

    rng = np.random.default_rng(0x5EED0000 + A.n)
    for k in (1, 3, 17):
        B = rng.standard_normal((A.n, k)) if k > 1 else rng.standard_normal(A.n)
        X = chol.Solve(B)
        Xo = ref.solve(B)
        assert rel_err(X, Xo) < sol_tol, k
        assert backward_error(A, X, B, reg) < 1e-14, k
        assert backward_error(A, Xo, B, reg) < 1e-14, k

    assert abs(chol.LogDeterminant() - ref.log_det()) <= 1e-10 * max(1.0, abs(ref.log_det()))


def test_many_rhs_alpha_beta_and_leading_dimensions():
    A = M.grid_laplacian_2d(24, 0.0)
    perm = O.nested_dissection(A, 8)
    chol = CholeskyDecomposition(A.outer, A.inner, perm)
    ref = oracle.OracleCholesky(A.n, A.outer, A.inner, perm)
    assert chol.NumericFactorization(A.values, 0.5) == 0
    ref.factor(A.values, 0.5)
    rng = np.random.default_rng(3)
    k = 70                                      # more than one 64-column solve block
    B = rng.standard_normal((A.n, k))
    assert rel_err(chol.Solve(B), ref.solve(B)) < TOL

    # X = alpha A^{-1} B + beta X with ldB = ldX = 9 > nrhs = 5 (Solve.hpp:22)
    nrhs, ld = 5, 9
    Bw = rng.standard_normal((A.n, ld))
    Xw = rng.standard_normal((A.n, ld))
    X0 = Xw.copy()
    alpha, beta = -0.75, 2.5
    st = lib().tb_chol_solve(chol.handle, alpha, Bw.ctypes.data, ld, beta, Xw.ctypes.data, ld, nrhs)
    assert st == 0
    expect = alpha * ref.solve(np.ascontiguousarray(Bw[:, :nrhs])) + beta * X0[:, :nrhs]
    assert rel_err(Xw[:, :nrhs], expect) < TOL
    assert np.array_equal(Xw[:, nrhs:], X0[:, nrhs:])   # columns beyond nrhs untouched

    # beta == 0 must not read X (NaNs there are overwritten)
    Xn = np.full((A.n, 3), np.nan)
    Bn = rng.standard_normal((A.n, 3))
    chol.Solve(Bn, Xn, alpha=1.0, beta=0.0)
    assert np.isfinite(Xn).all()

    # B and X may alias (Solve.hpp:43)
    Ba = rng.standard_normal((A.n, 4))
    expect = ref.solve(Ba)
    chol.Solve(Ba, Ba)
    assert rel_err(Ba, expect) < TOL


def test_half_solves_match_oracle():
    A = M.grid_laplacian_2d(16, 0.0)
    perm = O.nested_dissection(A, 8)
    chol = CholeskyDecomposition(A.outer, A.inner, perm)
    ref = oracle.OracleCholesky(A.n, A.outer, A.inner, perm)
    chol.NumericFactorization(A.values, 1e-1)
    ref.factor(A.values, 1e-1)
    B = np.random.default_rng(4).standard_normal((A.n, 2))
    assert rel_err(chol.UpperSolve(B), ref.solve(B, which="upper")) < TOL
    assert rel_err(chol.LowerSolve(B), ref.solve(B, which="lower")) < TOL
    # lower then upper is the full solve
    y = chol.LowerSolve(B)
    x = chol.UpperSolve(y)
    assert rel_err(x, chol.Solve(B)) < TOL


def test_not_positive_definite_is_reported():
    A = M.grid_laplacian_2d(10, 0.0)
    perm = O.nested_dissection(A, 8)
    chol = CholeskyDecomposition(A.outer, A.inner, perm)
    chol.SymbolicFactorization()
    # make the last pivot negative: it lies in the root supernode (n0 > 1),
    # where a non-positive pivot is reported (Multifrontal.hpp:445-449)
    last = int(chol.GetPermutation()[-1])
    rows = np.repeat(np.arange(A.n), np.diff(A.outer))
    vals = A.values.copy()
    vals[np.where((rows == last) & (A.inner == last))[0][0]] = -100.0
    ref = oracle.OracleCholesky(A.n, A.outer, A.inner, perm)
    assert ref.factor(vals, 0.0) == 1
    assert chol.NumericFactorization(vals, 0.0) == 1   # Numeric.hpp:99
    assert chol.NumericallyFactorizedQ() and not chol.NumericallyGoodQ()
    assert chol.FailedSupernode() == chol.SN_Count() - 1
    with pytest.raises(TBError):
        chol.Solve(np.ones(A.n))
    # a good matrix afterwards factors again
    assert chol.NumericFactorization(A.values, 1e-2) == 0
    assert chol.NumericallyGoodQ()


def test_negative_one_by_one_pivot_follows_reference():
    # Arrow matrix [[a,0,x],[0,b,y],[x,y,c]]: with the Fundamental strategy
    # every row is its own 1 x 1 supernode, and the reference takes sqrt(|a|)
    # for a 1 x 1 pivot without reporting failure (Multifrontal.hpp:471).
    outer = np.array([0, 2, 4, 7], dtype=np.int64)
    inner = np.array([0, 2, 1, 2, 0, 1, 2], dtype=np.int32)
    vals = np.array([-4.0, 1.0, 9.0, 1.0, 1.0, 1.0, 100.0])
    chol = CholeskyDecomposition(outer, inner)
    chol.SetSupernodeStrategy(1)
    ref = oracle.OracleCholesky(3, outer, inner, None, "fundamental")
    assert list(chol.SN_RowPointers()) == list(ref.array("SN_rp")) == [0, 1, 2, 3]
    assert ref.factor(vals) == 0
    assert chol.NumericFactorization(vals) == 0
    tri, rec = chol.FactorValues()
    to, ro = ref.factor_values()
    assert np.allclose(tri, to) and np.allclose(rec, ro) and tri[0] == 2.0


def test_diagonal_matrix_is_one_supernode_like_the_reference():
    # No row of a diagonal matrix starts a fundamental supernode
    # (Symbolic.hpp:590-622), so all rows form one dense supernode and a
    # negative entry is a failed pivot, as in the reference.
    n = 7
    outer = np.arange(n + 1, dtype=np.int64)
    inner = np.arange(n, dtype=np.int32)
    vals = np.array([4.0, -9.0, 1.0, 2.0, -1.0, 16.0, 3.0])
    chol = CholeskyDecomposition(outer, inner)
    ref = oracle.OracleCholesky(n, outer, inner)
    assert chol.SN_Count() == ref.sn_count() == 1
    assert chol.NumericFactorization(vals) == ref.factor(vals) == 1
    assert chol.NumericFactorization(np.abs(vals)) == 0
    assert np.allclose(chol.WriteFactorDiagonal(), np.sqrt(np.abs(vals)))


def test_single_row_and_two_by_two():
    outer = np.array([0, 1], dtype=np.int64)
    inner = np.array([0], dtype=np.int32)
    chol = CholeskyDecomposition(outer, inner)
    assert chol.NumericFactorization(np.array([4.0])) == 0
    assert np.allclose(chol.Solve(np.array([2.0])), [0.5])
    outer = np.array([0, 2, 4], dtype=np.int64)
    inner = np.array([0, 1, 0, 1], dtype=np.int32)
    vals = np.array([4.0, 2.0, 2.0, 3.0])
    chol = CholeskyDecomposition(outer, inner, np.array([1, 0], dtype=np.int32))
    assert chol.NumericFactorization(vals) == 0
    b = np.array([1.0, 2.0])
    assert np.allclose(chol.Solve(b), np.linalg.solve(vals.reshape(2, 2), b))


@pytest.mark.parametrize("grid,leaf,schedule", [(10, 16, "task_graph_all"), (24, 64, "task_graph"),
                                                (18, 8, "task_graph_all"), (28, 32, "task_graph")])
def test_task_graph_and_level_schedules_agree_bitwise(grid, leaf, schedule):
    # the persistent task-graph launch runs the same task bodies in a
    # dependency order; every entry is produced by the same sequence of
    # floating-point operations, so the factors are identical
    A = M.grid_laplacian_3d(grid, 12, 1e-3)
    perm = O.nested_dissection(A, leaf)
    a = CholeskyDecomposition(A.outer, A.inner, perm)
    b = CholeskyDecomposition(A.outer, A.inner, perm)
    a.SetSchedule(schedule)
    b.SetSchedule("levels")
    for _ in range(2):
        assert a.NumericFactorization(A.values) == 0
        assert b.NumericFactorization(A.values) == 0
        ta, ra = a.FactorValues()
        tb_, rb = b.FactorValues()
        assert np.array_equal(ta, tb_) and np.array_equal(ra, rb)
    B = np.random.default_rng(grid).standard_normal((A.n, 3))
    xa, xb = a.Solve(B), b.Solve(B)
    assert rel_err(xa, xb) < 1e-12


@pytest.mark.parametrize("grid,leaf,nrhs", [(24, 64, 1), (28, 32, 16), (16, 8, 70)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_solve_task_graph_matches_level_launches(grid, leaf, nrhs, precision):
    # the persistent solve runs the same step bodies in dependency order; rows
    # shared between tasks are updated by atomic additions in another order, so
    # the sweeps agree to rounding, and every schedule solves the system
    A = M.grid_laplacian_3d(grid, 14, 1e-3)
    perm = O.nested_dissection(A, leaf)
    c = CholeskyDecomposition(A.outer, A.inner, perm)
    c.SetPrecision(precision)
    c.SetRefinement(1e-12, 30)
    assert c.NumericFactorization(A.values) == 0
    B = np.random.default_rng(grid + nrhs).standard_normal((A.n, nrhs))
    out = {}
    for sched in ("levels", "task_graph", "task_graph_all", "levels"):
        c.SetSolveSchedule(sched)
        out[sched] = (c.Solve(B), c.UpperSolve(B), c.LowerSolve(B))
    ref = out["levels"]
    S = A.to_scipy()
    for sched in ("task_graph", "task_graph_all"):
        # the refined mixed solve iterates from slightly different preconditioner
        # outputs, so its result agrees to the refinement target instead
        tols = (1e-12 if precision == "fp64" else 1e-8, 1e-12, 1e-12)
        for got, want, tol in zip(out[sched], ref, tols):
            assert rel_err(got, want) < tol, sched
        X = out[sched][0]
        R = B - S @ X
        assert np.max(np.linalg.norm(R, axis=0) / np.linalg.norm(B, axis=0)) < 1e-10


def test_solve_task_graph_without_device_allocation():
    torch = pytest.importorskip("torch")
    A = M.grid_laplacian_3d(20, 15, 1e-3)
    perm = O.nested_dissection(A, 32)
    c = CholeskyDecomposition(A.outer, A.inner, perm)
    assert c.NumericFactorization(A.values) == 0
    from tensors_b200 import _lib

    lib = _lib.lib()
    k = 4
    B = torch.tensor(np.random.default_rng(3).standard_normal((A.n, k)), device="cuda")
    c.SetSolveSchedule("levels")
    X_lv = torch.zeros_like(B)
    assert lib.tb_chol_solve_device(c.handle, 1.0, B.data_ptr(), k, 0.0, X_lv.data_ptr(), k, k) == 0
    torch.cuda.synchronize()
    c.SetSolveSchedule("task_graph")
    X = torch.full_like(B, float("nan"))
    assert lib.tb_chol_solve_device_noalloc(c.handle, 1.0, B.data_ptr(), k, 0.0, X.data_ptr(), k, k) == 0
    torch.cuda.synchronize()
    assert rel_err(X.cpu().numpy(), X_lv.cpu().numpy()) < 1e-12


def test_autotune_keeps_the_factor_and_the_solution():
    A = M.grid_laplacian_3d(20, 16, 1e-3)
    perm = O.nested_dissection(A, 32)
    c = CholeskyDecomposition(A.outer, A.inner, perm)
    assert c.NumericFactorization(A.values) == 0
    tri0, rec0 = c.FactorValues()
    B = np.random.default_rng(16).standard_normal((A.n, 4))
    X0 = c.Solve(B)
    r = c.Autotune(4)
    assert r["factor"] in ("levels", "task_graph") and r["solve"] in ("levels", "task_graph")
    assert all(np.isfinite(v) and v > 0 for v in r["times_ms"].values()), r
    # the chosen factor schedule is kept: refactoring gives the same factor, bit for bit
    tri, rec = c.FactorValues()
    assert np.array_equal(tri, tri0) and np.array_equal(rec, rec0)
    assert c.NumericFactorization(A.values) == 0
    tri, rec = c.FactorValues()
    assert np.array_equal(tri, tri0) and np.array_equal(rec, rec0)
    assert rel_err(c.Solve(B), X0) < 1e-12


def test_graph_and_direct_launches_agree_bitwise():
    A = M.grid_laplacian_3d(10, 11, 1e-3)
    perm = O.nested_dissection(A, 16)
    a = CholeskyDecomposition(A.outer, A.inner, perm)
    b = CholeskyDecomposition(A.outer, A.inner, perm)
    b.SetUseGraph(False)
    a.NumericFactorization(A.values)
    b.NumericFactorization(A.values)
    ta, ra = a.FactorValues()
    tb_, rb = b.FactorValues()
    assert np.array_equal(ta, tb_) and np.array_equal(ra, rb)
    # refactoring with the captured graph reproduces the factor exactly
    a.NumericFactorization(A.values)
    t2, r2 = a.FactorValues()
    assert np.array_equal(ta, t2) and np.array_equal(ra, r2)


def test_device_buffers_and_residual():
    torch = pytest.importorskip("torch")
    A = M.grid_laplacian_2d(30, 0.0)
    perm = O.nested_dissection(A, 8)
    chol = CholeskyDecomposition(A.outer, A.inner, perm)
    vals = torch.tensor(A.values, device="cuda", dtype=torch.float64)
    assert chol.NumericFactorization(vals, 1e-2) == 0
    B = torch.randn(A.n, 6, device="cuda", dtype=torch.float64)
    X = chol.Solve(B)
    ref = oracle.OracleCholesky(A.n, A.outer, A.inner, perm)
    ref.factor(A.values, 1e-2)
    assert rel_err(X.cpu().numpy(), ref.solve(B.cpu().numpy())) < TOL
    # the residual kernel uses the caller-order matrix without the shift
    R = chol.Residual(B, X).cpu().numpy()
    expect = B.cpu().numpy() - A.to_scipy() @ X.cpu().numpy()
    assert rel_err(R, expect) < 1e-12


def test_factor_diagonal_and_reference_layout_export():
    A = M.delaunay_laplacian(1500, 21)
    perm = O.nested_dissection(A, 16)
    chol = CholeskyDecomposition(A.outer, A.inner, perm)
    chol.NumericFactorization(A.values, 0.0)
    d = chol.WriteFactorDiagonal()
    tri, _ = chol.FactorValues()
    rp, tp = chol.SN_RowPointers(), chol.SN_TrianglePointers()
    expect = np.concatenate([np.diag(tri[tp[s]:tp[s + 1]].reshape(rp[s + 1] - rp[s], -1)) for s in range(len(rp) - 1)])
    assert np.array_equal(d, expect)
    # U^T U reproduces P A P^T
    U = chol.GetU().toarray()
    p = chol.GetPermutation()
    S = A.to_scipy().toarray()[np.ix_(p, p)]
    assert np.abs(U.T @ U - S).max() < 1e-10 * np.abs(S).max()


def test_get_u_through_the_c_abi_matches_the_python_assembly():
    A = M.delaunay_laplacian(1200, 23)
    chol = CholeskyDecomposition(A.outer, A.inner, O.nested_dissection(A, 16))
    assert chol.NumericFactorization(A.values, 0.0) == 0
    nnz = chol.UNonzeroCount()
    outer = np.zeros(A.n + 1, dtype=np.int64)
    inner = np.zeros(nnz, dtype=np.int32)
    values = np.zeros(nnz)
    assert lib().tb_chol_get_u(chol._h, outer.ctypes.data, inner.ctypes.data, values.ctypes.data) == 0
    U = chol.GetU()
    U.sort_indices()
    assert np.array_equal(outer, U.indptr) and np.array_equal(inner, U.indices) and np.array_equal(values, U.data)


def test_left_looking_setting_gives_the_multifrontal_factor_bitwise():
    from tensors_b200.cholesky import FactorizationMethod

    A = M.delaunay_laplacian(1500, 4)
    perm = O.nested_dissection(A, 16)
    vals = []
    for method in (FactorizationMethod.Multifrontal, FactorizationMethod.LeftLooking):
        c = CholeskyDecomposition(A.outer, A.inner, perm)
        c.SetFactorizationMethod(method)
        assert c.NumericFactorization(A.values, 1e-3) == 0
        vals.append(c.FactorValues())
    for a, b in zip(*vals):
        assert np.array_equal(a, b)
