"""Batches of independent systems (tb_batch_*): one block-diagonal matrix,
one persistent factorization launch, per-system results identical to
factoring each system alone."""
from __future__ import annotations

import numpy as np
import pytest

from tensors_b200 import matrices as M
from tensors_b200 import ordering as O
from tensors_b200.cholesky import BatchedCholesky, CholeskyDecomposition


def _systems(count=12, seed=7):
    rng = np.random.default_rng(seed)
    out = []
    for s in range(count):
        kind = s % 3
        if kind == 0:
            A = M.delaunay_laplacian(int(rng.integers(200, 1500)), 100 + s)
        elif kind == 1:
            A = M.grid_laplacian_2d(int(rng.integers(5, 30)), 1e-2)
        else:
            A = M.grid_laplacian_3d(int(rng.integers(4, 11)), 200 + s, 1e-2)
        perm = O.nested_dissection(A, 16) if s % 4 != 3 else None
        out.append((A, perm))
    return out


SYSTEMS = _systems()


def test_batch_symbolic_keeps_systems_contiguous():
    b = BatchedCholesky([(A.outer, A.inner, p) for A, p in SYSTEMS])
    perm = b.handle.GetPermutation()
    sn = 0
    for s, (A, p) in enumerate(SYSTEMS):
        r0, r1 = b.row_offsets[s], b.row_offsets[s + 1]
        c = CholeskyDecomposition(A.outer, A.inner, p)
        assert np.array_equal(perm[r0:r1] - r0, c.GetPermutation())
        sn += c.SN_Count()
    assert b.handle.SN_Count() == sn
    assert b.handle.NonzeroCount() == sum(len(A.inner) for A, _ in SYSTEMS)


@pytest.mark.gpu
def test_batch_factor_and_solve_match_single_systems():
    b = BatchedCholesky([(A.outer, A.inner, p) for A, p in SYSTEMS])
    assert b.NumericFactorization([A.values for A, _ in SYSTEMS], 0.0) == 0
    assert b.FailedSystem() == -1
    Bs = [np.random.default_rng(s).standard_normal(A.n) for s, (A, _) in enumerate(SYSTEMS)]
    Xs = b.Solve(Bs)
    t_all, r_all = b.handle.FactorValues()
    tp, rp = b.handle.SN_TrianglePointers(), b.handle.SN_RectanglePointers()
    sn0 = 0
    for s, (A, p) in enumerate(SYSTEMS):
        c = CholeskyDecomposition(A.outer, A.inner, p)
        assert c.NumericFactorization(A.values, 0.0) == 0
        t, r = c.FactorValues()
        S = c.SN_Count()
        # the system's supernodes are a contiguous run of the batch's, with identical values
        assert np.array_equal(t_all[tp[sn0]:tp[sn0 + S]], t)
        assert np.array_equal(r_all[rp[sn0]:rp[sn0 + S]], r)
        sn0 += S
        x = c.Solve(Bs[s])
        assert np.abs(Xs[s] - x).max() <= 1e-12 * np.abs(x).max()


@pytest.mark.gpu
def test_batch_mixed_precision_and_device_buffers():
    import torch

    vals = torch.tensor(np.concatenate([A.values for A, _ in SYSTEMS]), device="cuda")
    B = torch.randn(int(b_rows := sum(A.n for A, _ in SYSTEMS)), dtype=torch.float64, device="cuda",
                    generator=torch.Generator(device="cuda").manual_seed(5))
    # some Delaunay systems here have kappa ~1e10: the target is 1e-10 or what the
    # FP64 direct solve of the same batch attains, whichever is larger
    ref = BatchedCholesky([(A.outer, A.inner, p) for A, p in SYSTEMS])
    assert ref.NumericFactorization(vals, 0.0) == 0
    X64 = ref.Solve(B)
    torch.cuda.synchronize()
    X64 = X64.cpu().numpy()
    Bh = B.cpu().numpy()

    def relres(X):
        # residual of the whole block-diagonal system, as the refinement measures it
        R = np.concatenate([Bh[ref.row_offsets[s]:ref.row_offsets[s + 1]]
                            - A.to_scipy() @ X[ref.row_offsets[s]:ref.row_offsets[s + 1]]
                            for s, (A, _) in enumerate(SYSTEMS)])
        return np.linalg.norm(R) / np.linalg.norm(Bh)

    target = max(1e-10, 4.0 * relres(X64))
    b = BatchedCholesky([(A.outer, A.inner, p) for A, p in SYSTEMS])
    b.handle.SetPrecision("mixed")
    b.handle.SetRefinement(target, 100)
    assert b.NumericFactorization(vals, 0.0) == 0
    X = b.Solve(B)
    torch.cuda.synchronize()
    it, rr = b.handle.RefinementInfo()
    assert rr <= target and it >= 1, (rr, it, target)
    assert relres(X.cpu().numpy()) <= 2 * target, (relres(X.cpu().numpy()), target)
    assert b_rows == int(b.row_offsets[-1])


@pytest.mark.gpu
def test_batch_reports_the_failing_system():
    systems = SYSTEMS[:6]
    vals = [A.values.copy() for A, _ in systems]
    A4 = systems[4][0]
    d = np.repeat(np.arange(A4.n), np.diff(A4.outer)) == A4.inner
    vals[4][d] -= 100.0                                   # system 4 indefinite
    b = BatchedCholesky([(A.outer, A.inner, p) for A, p in systems])
    assert b.NumericFactorization(vals, 0.0) == 1
    assert b.FailedSystem() == 4
