"""Seeded fuzzing of the host boundary (no GPU): corrupted patterns and
permutations through the constructor (single systems and batches), symbolic
analysis, plan and plan check;
mutated MatrixMarket files through the reader; adversarial graphs through the
pattern-only nested dissection.  Every input either works or fails with a
status (TBError); nothing crashes, and what is accepted is consistent."""
from __future__ import annotations

import numpy as np

from tensors_b200 import matrices as M
from tensors_b200 import ordering as O
from tensors_b200.cholesky import CholeskyDecomposition, TBError
from tensors_b200.matrix_market import read_matrix_market, write_matrix_market


def test_corrupted_patterns_and_permutations():
    rng = np.random.default_rng(3)
    A = M.grid_laplacian_2d(9, 1.0)
    base_perm = O.nested_dissection(A, 8)
    rejected = 0
    for _ in range(400):
        outer, inner, perm = A.outer.copy(), A.inner.copy(), base_perm.copy()
        kind = rng.integers(0, 6)
        if kind == 0:
            inner[rng.integers(0, len(inner))] = rng.integers(-5, A.n + 5)
        elif kind == 1:
            outer[rng.integers(1, len(outer))] += rng.integers(-3, 4)
        elif kind == 2:
            perm[rng.integers(0, len(perm))] = rng.integers(-2, A.n + 2)
        elif kind == 3:
            k = rng.integers(0, len(inner) - 1)
            inner[k], inner[k + 1] = inner[k + 1], inner[k]
        elif kind == 4:
            inner = inner[: rng.integers(0, len(inner))]
            outer = np.minimum(outer, len(inner))
        else:
            perm = None
        try:
            c = CholeskyDecomposition(outer, inner, perm)
            c.SymbolicFactorization()
            c.CheckPlan()
        except TBError:
            rejected += 1
    assert 0 < rejected < 400


def test_mutated_matrix_market_files(tmp_path):
    rng = np.random.default_rng(4)
    A = M.grid_laplacian_2d(8, 1.0)
    base = tmp_path / "base.mtx"
    write_matrix_market(base, A)
    data = base.read_bytes()
    rejected = 0
    for t in range(400):
        d = bytearray(data)
        for _ in range(rng.integers(1, 8)):
            d[int(rng.integers(0, len(d)))] = int(rng.integers(0, 256))
        if rng.random() < 0.2:
            d = d[: int(rng.integers(0, len(d)))]
        f = tmp_path / "t.mtx"
        f.write_bytes(bytes(d))
        try:
            m, n, outer, inner, values = read_matrix_market(f)
        except TBError:
            rejected += 1
            continue
        assert len(outer) == m + 1 and outer[-1] == len(inner) == len(values)
        assert len(inner) == 0 or (inner.min() >= 0 and inner.max() < n)
        assert np.all(np.diff(outer) >= 0)
    assert 0 < rejected < 400


def _symmetric(n, rows, cols):
    r = np.concatenate([rows, cols, np.arange(n)])
    c = np.concatenate([cols, rows, np.arange(n)])
    return M.from_coo(n, r, c, np.ones(len(r)))


def test_adversarial_graphs_are_ordered():
    rng = np.random.default_rng(5)
    n = 3000
    i, j = np.triu_indices(120, 1)
    graphs = [
        _symmetric(n, np.zeros(n - 1, np.int64), np.arange(1, n)),                       # star
        _symmetric(30000, np.arange(29999), np.arange(1, 30000)),                         # path
        _symmetric(120, i, j),                                                            # clique
        _symmetric(20000, rng.integers(0, 20000, 60000), rng.integers(0, 20000, 60000)),  # random
        _symmetric(20000, np.arange(0, 20000, 2), np.arange(1, 20000, 2)),                # pairs
        _symmetric(25000, np.zeros(0, np.int64), np.zeros(0, np.int64)),                  # diagonal
    ]
    for G in graphs:
        p = O.graph_nested_dissection(G, 64)
        assert O.is_permutation(p, G.n)
        assert np.array_equal(p, O.graph_nested_dissection(G, 64, thread_count=1))


def test_corrupted_systems_in_a_batch():
    from tensors_b200.cholesky import BatchedCholesky

    rng = np.random.default_rng(6)
    mats = [M.grid_laplacian_2d(int(g), 1.0) for g in (3, 5, 7, 4)]
    rejected = 0
    for _ in range(200):
        systems = []
        for A in mats:
            outer, inner, perm = A.outer.copy(), A.inner.copy(), O.nested_dissection(A, 8).copy()
            if rng.random() < 0.3:
                kind = rng.integers(0, 3)
                if kind == 0:
                    inner[rng.integers(0, len(inner))] = rng.integers(-3, A.n + 3)
                elif kind == 1:
                    perm[rng.integers(0, len(perm))] = rng.integers(-2, A.n + 2)
                else:
                    outer[rng.integers(1, len(outer))] += rng.integers(-2, 3)
            systems.append((outer, inner, perm))
        try:
            b = BatchedCholesky(systems)
            b.handle.SymbolicFactorization()
            b.handle.CheckPlan()
        except TBError:
            rejected += 1
    assert 0 < rejected < 200
