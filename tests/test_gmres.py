"""GMRES preconditioned by the GPU factor (tb_chol_gmres / _device), and GMRES-IR inside the
mixed-precision solve.

Checked against a numpy restatement of the reference's ``GMRES::operator()`` (GMRES.hpp:124-655:
left preconditioning, two Gram-Schmidt passes, Givens rotations, restarts) whose preconditioner is
the oracle's factor solve: the same iteration counts (to rounding), the reference's stopping rule
|P r| <= tol |P b| met, and solutions that agree.  GMRES-IR: a mixed-precision handle whose CG
refinement is denied every step reaches the target through GMRES on the FP64 system."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from tensors_b200 import matrices as M
from tensors_b200 import ordering as O
from tensors_b200.cholesky import CholeskyDecomposition

pytestmark = pytest.mark.gpu


def _gmres_restatement(A, P, B, tol, m, max_restarts):
    """GMRES.hpp:124-655 (left preconditioned, per column), sign convention r = b - A x."""
    n, k = B.shape
    x = np.zeros_like(B)
    bn = np.linalg.norm(P(B), axis=0)
    TOL = tol * bn
    total = 0
    for restart in range(max_restarts + 1):
        r = P(B - M.csr_matvec(A, x)) if restart or x.any() else P(B)
        beta0 = np.linalg.norm(r, axis=0)
        Q = [r / beta0]
        H = np.zeros((m + 1, m, k))
        cs, sn = np.zeros((m, k)), np.zeros((m, k))
        beta = np.zeros((m + 1, k))
        beta[0] = beta0
        it = 0
        succ = np.all(beta0 <= TOL)
        while not succ and it < m:
            q = P(M.csr_matvec(A, Q[it]))
            for _ in range(2):
                hcol = np.array([np.sum(Qi * q, axis=0) for Qi in Q])
                q = q - sum(hcol[i] * Q[i] for i in range(len(Q)))
                H[: it + 1, it] += hcol
            qn = np.linalg.norm(q, axis=0)
            H[it + 1, it] = qn
            Q.append(q / qn)
            for i in range(it):
                xi, eta = H[i, it].copy(), H[i + 1, it].copy()
                H[i, it] = cs[i] * xi + sn[i] * eta
                H[i + 1, it] = -sn[i] * xi + cs[i] * eta
            xi, eta = H[it, it].copy(), H[it + 1, it].copy()
            rr = np.sqrt(xi * xi + eta * eta)
            cs[it] = np.abs(xi) / rr
            sn[it] = np.sign(xi) * eta / rr
            H[it, it] = cs[it] * xi + sn[it] * eta
            H[it + 1, it] = 0.0
            beta[it + 1] = -sn[it] * beta[it]
            beta[it] = cs[it] * beta[it]
            it += 1
            succ = np.all(np.abs(beta[it]) <= TOL)
        for c in range(k):
            y = np.linalg.solve(np.triu(H[:it, :it, c]), beta[:it, c]) if it else np.zeros(0)
            x[:, c] += sum(y[j] * Q[j][:, c] for j in range(it))
        total += it
        if succ:
            return x, total, restart, True
    return x, total, max_restarts, False


def _nearby_pair(g=18):
    A = M.grid_laplacian_3d(g, 51, 1e-3)
    d = 1.0 + 0.2 * np.random.default_rng(52).uniform(-1.0, 1.0, A.n)
    rows = np.repeat(np.arange(A.n), np.diff(A.outer))
    A2 = M.CSRMatrix(n=A.n, outer=A.outer, inner=A.inner, values=d[rows] * A.values * d[A.inner])
    return A, A2, O.nested_dissection(A, 16)


def test_gmres_on_a_nearby_matrix_matches_the_restatement():
    A, A2, perm = _nearby_pair()
    c = CholeskyDecomposition(A.outer, A.inner, perm)
    assert c.NumericFactorization(A.values) == 0
    o = oracle.OracleCholesky(A.n, A.outer, A.inner, perm)
    assert o.factor(A.values) == 0
    B = np.random.default_rng(53).standard_normal((A.n, 3))
    X, ok = c.GMRES(B, values=A2.values, relative_tolerance=1e-10, max_iter=20, max_restarts=10)
    assert ok
    x_ref, it_ref, rs_ref, ok_ref = _gmres_restatement(A2, lambda R: o.solve(R), B, 1e-10, 20, 10)
    assert ok_ref and it_ref > 3
    assert abs(c.IterationCount() - it_ref) <= 1 and c.GMRESRestarts() == rs_ref
    assert np.all(c.RelativeResiduals() <= 1e-10)
    assert np.linalg.norm(X - x_ref) <= 1e-7 * np.linalg.norm(x_ref)
    S = A2.to_scipy()
    assert np.linalg.norm(B - S @ X) / np.linalg.norm(B) <= 1e-8


def test_gmres_device_equals_host_and_alpha_beta():
    import torch

    A, A2, perm = _nearby_pair(12)
    c = CholeskyDecomposition(A.outer, A.inner, perm)
    assert c.NumericFactorization(A.values) == 0
    B = np.random.default_rng(54).standard_normal((A.n, 2))
    Xh, ok = c.GMRES(B, values=A2.values, relative_tolerance=1e-11, max_iter=20)
    assert ok
    Bd = torch.tensor(B, device="cuda")
    X0 = torch.tensor(np.random.default_rng(55).standard_normal((A.n, 2)), device="cuda")
    Xd = X0.clone()
    _, ok = c.GMRES(Bd, Xd, values=torch.tensor(A2.values, device="cuda"), alpha=2.0, beta=-1.0,
                    relative_tolerance=1e-11, max_iter=20)
    assert ok
    expect = 2.0 * Xh - X0.cpu().numpy()
    assert np.abs(Xd.cpu().numpy() - expect).max() <= 1e-9 * np.abs(expect).max()


def test_gmres_ir_rescues_a_refinement_that_cannot_converge():
    """The refinement's CG is limited to 0 steps: the mixed solve then needs GMRES-IR (not the FP64 refactor)."""
    A = M.vector_laplacian_3d(10, 0x5EED0056, 1e-2)
    c = CholeskyDecomposition(A.outer, A.inner, O.nested_dissection(A))
    c.SetPrecision("mixed")
    c.SetRefinement(1e-12, 0)
    assert c.NumericFactorization(A.values, 0.0) == 0
    B = np.random.default_rng(56).standard_normal((A.n, 4))
    X = c.Solve(B)
    assert c.GMRESIRIterations() > 0
    assert c.PrecisionInUse() == ("mixed", False)          # no FP64 refactorization
    S = A.to_scipy()
    assert np.linalg.norm(B - S @ X) / np.linalg.norm(B) <= 1e-12
