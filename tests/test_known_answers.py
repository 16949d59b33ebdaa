"""Known-answer tests of the oracle (closed forms and tiny hand cases)."""
from __future__ import annotations

import numpy as np

import oracle
from tensors_b200 import matrices as M


def test_tridiagonal_closed_form():
    # T = tridiag(-1, 2, -1): U(k,k) = sqrt((k+2)/(k+1)), U(k,k+1) = -sqrt((k+1)/(k+2)),
    # det T = n + 1.
    n = 40
    rows = np.concatenate([np.arange(n), np.arange(n - 1), np.arange(1, n)])
    cols = np.concatenate([np.arange(n), np.arange(1, n), np.arange(n - 1)])
    vals = np.concatenate([np.full(n, 2.0), np.full(n - 1, -1.0), np.full(n - 1, -1.0)])
    A = M.from_coo(n, rows, cols, vals)
    o = oracle.OracleCholesky(n, A.outer, A.inner)
    assert o.factor(A.values) == 0
    k = np.arange(n)
    U = np.zeros((n, n))
    rp, so, si = o.array("SN_rp"), o.array("SN_outer"), o.array("SN_inner")
    tp, rcp = o.array("SN_tri_ptr"), o.array("SN_rec_ptr")
    tri, rec = o.factor_values()
    for s in range(len(rp) - 1):
        i0, n0, n1 = rp[s], rp[s + 1] - rp[s], so[s + 1] - so[s]
        U[i0:i0 + n0, i0:i0 + n0] = tri[tp[s]:tp[s] + n0 * n0].reshape(n0, n0)
        if n1:
            U[np.ix_(np.arange(i0, i0 + n0), si[so[s]:so[s + 1]])] = rec[rcp[s]:rcp[s] + n0 * n1].reshape(n0, n1)
    assert np.allclose(np.diag(U), np.sqrt((k + 2) / (k + 1)))
    assert np.allclose(np.diag(U, 1), -np.sqrt((k[:-1] + 1) / (k[:-1] + 2)))
    assert np.isclose(o.log_det(), np.log(n + 1))


def test_two_by_two_by_hand():
    # [[4,2],[2,3]] = U^T U with U = [[2,1],[0,sqrt(2)]]
    outer = np.array([0, 2, 4], dtype=np.int64)
    inner = np.array([0, 1, 0, 1], dtype=np.int32)
    o = oracle.OracleCholesky(2, outer, inner)
    assert o.factor(np.array([4.0, 2.0, 2.0, 3.0])) == 0
    tri, rec = o.factor_values()
    U = np.zeros((2, 2))
    if len(tri) == 4:
        U = tri.reshape(2, 2)
    assert np.allclose(U, [[2.0, 1.0], [0.0, np.sqrt(2.0)]])
    assert np.allclose(o.solve(np.array([8.0, 7.0])), np.linalg.solve([[4, 2], [2, 3]], [8.0, 7.0]))


def test_diagonal_and_shift():
    n = 5
    outer = np.arange(n + 1, dtype=np.int64)
    inner = np.arange(n, dtype=np.int32)
    d = np.array([1.0, 4.0, 9.0, 16.0, 25.0])
    o = oracle.OracleCholesky(n, outer, inner)
    assert o.factor(d, reg=0.5) == 0      # reg is added to every diagonal entry (Multifrontal.hpp:274)
    b = np.ones(n)
    assert np.allclose(o.solve(b), b / (d + 0.5))
    assert np.isclose(o.log_det(), np.log(d + 0.5).sum())


def test_indefinite_reported():
    outer = np.array([0, 2, 4], dtype=np.int64)
    inner = np.array([0, 1, 0, 1], dtype=np.int32)
    o = oracle.OracleCholesky(2, outer, inner)
    assert o.factor(np.array([1.0, 2.0, 2.0, 1.0])) == 1
