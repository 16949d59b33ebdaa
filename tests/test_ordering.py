"""Nested-dissection orderings (geometric, and from the pattern alone): validity and fill reduction."""
from __future__ import annotations

import numpy as np
import pytest

from tensors_b200 import matrices as M
from tensors_b200 import ordering as O
from tensors_b200.cholesky import CholeskyDecomposition, TBError


def test_nested_dissection_is_a_permutation():
    for A in (M.grid_laplacian_2d(37, 1.0), M.grid_laplacian_3d(11, 1), M.vector_laplacian_3d(4, 1),
              M.delaunay_laplacian(1000, 2)):
        p = O.nested_dissection(A)
        assert O.is_permutation(p, A.n)
        if A.dofs_per_node > 1:        # the dofs of a node stay together
            assert np.array_equal(p.reshape(-1, 3) // 3, np.repeat((p[::3] // 3)[:, None], 3, axis=1))


def test_nested_dissection_reduces_fill():
    A = M.grid_laplacian_2d(40, 1.0)
    nat = CholeskyDecomposition(A.outer, A.inner, O.identity_ordering(A.n)).FlopCount()[1]
    nd = CholeskyDecomposition(A.outer, A.inner, O.nested_dissection(A)).FlopCount()[1]
    assert nd < 0.6 * nat


# ---------------------------------------------------------------- graph nested dissection


def _flops(A, p):
    return CholeskyDecomposition(A.outer, A.inner, p).FlopCount()[0]


def _upper_only(A):
    rows = np.repeat(np.arange(A.n), np.diff(A.outer))
    keep = A.inner >= rows
    outer = np.concatenate([[0], np.cumsum(np.bincount(rows[keep], minlength=A.n))]).astype(np.int64)
    return M.CSRMatrix(n=A.n, outer=outer, inner=A.inner[keep], values=A.values[keep], dofs_per_node=A.dofs_per_node)


def test_graph_nested_dissection_is_a_permutation():
    for A in (M.grid_laplacian_2d(37, 1.0), M.grid_laplacian_3d(11, 1), M.vector_laplacian_3d(4, 1),
              M.delaunay_laplacian(1000, 2)):
        p = O.graph_nested_dissection(A)
        assert O.is_permutation(p, A.n)
        assert np.array_equal(p, O.graph_nested_dissection(A))          # deterministic
        assert np.array_equal(p, O.graph_nested_dissection(A, thread_count=1))   # and the same on one thread
        if A.dofs_per_node > 1:
            assert np.array_equal(p.reshape(-1, 3), (p[::3] // 3)[:, None] * 3 + np.arange(3))


def test_graph_nested_dissection_edge_cases():
    # components: two disjoint grids in one matrix
    A = M.grid_laplacian_2d(20, 1.0)
    n = A.n
    two = M.CSRMatrix(n=2 * n, outer=np.concatenate([A.outer, A.outer[1:] + A.nnz]),
                      inner=np.concatenate([A.inner, A.inner + n]), values=np.concatenate([A.values, A.values]))
    assert O.is_permutation(O.graph_nested_dissection(two, 16), 2 * n)
    # one node, no rows, no diagonal entries, and one triangle of the pattern only
    one = M.CSRMatrix(n=1, outer=np.array([0, 1]), inner=np.array([0], np.int32), values=np.ones(1))
    assert np.array_equal(O.graph_nested_dissection(one), [0])
    empty = M.CSRMatrix(n=0, outer=np.zeros(1, np.int64), inner=np.zeros(0, np.int32), values=np.zeros(0))
    assert O.graph_nested_dissection(empty).shape == (0,)
    rows = np.repeat(np.arange(n), np.diff(A.outer))
    off = A.inner != rows
    nodiag = M.CSRMatrix(n=n, outer=np.concatenate([[0], np.cumsum(np.bincount(rows[off], minlength=n))]).astype(np.int64),
                         inner=A.inner[off], values=A.values[off])
    assert np.array_equal(O.graph_nested_dissection(nodiag), O.graph_nested_dissection(A))
    B = M.vector_laplacian_3d(5, 3)
    assert np.array_equal(O.graph_nested_dissection(_upper_only(B)), O.graph_nested_dissection(B))


def test_graph_nested_dissection_rejects_bad_input():
    A = M.grid_laplacian_2d(5, 1.0)
    with pytest.raises(TBError) as e:
        O.graph_nested_dissection(M.CSRMatrix(n=A.n, outer=A.outer, inner=A.inner, values=A.values, dofs_per_node=2))
    assert e.value.status == -1                      # 25 rows are not whole nodes of 2
    bad = A.inner.copy()
    bad[3] = A.n
    with pytest.raises(TBError) as e:
        O.graph_nested_dissection(M.CSRMatrix(n=A.n, outer=A.outer, inner=bad, values=A.values))
    assert e.value.status == -2


def test_graph_nested_dissection_fill():
    # measured against the geometric dissection (coordinates) and the natural order
    g2 = M.grid_laplacian_2d(60, 1.0)
    assert _flops(g2, O.graph_nested_dissection(g2)) < 0.3 * _flops(g2, O.identity_ordering(g2.n))       # 0.18
    g3 = M.grid_laplacian_3d(20, 4)
    assert _flops(g3, O.graph_nested_dissection(g3)) <= 0.8 * _flops(g3, O.nested_dissection(g3))        # 0.51
    mesh = M.delaunay_laplacian(5000, 6)
    assert _flops(mesh, O.graph_nested_dissection(mesh)) <= 2.0 * _flops(mesh, O.nested_dissection(mesh))  # 1.27
    vec = M.vector_laplacian_3d(8, 2)
    assert _flops(vec, O.graph_nested_dissection(vec)) <= 2.5 * _flops(vec, O.nested_dissection(vec))     # 1.31


def test_matrix_without_coordinates_is_ordered_from_its_pattern():
    A = M.delaunay_laplacian(3000, 8)
    bare = M.CSRMatrix(n=A.n, outer=A.outer, inner=A.inner, values=A.values)
    p = O.nested_dissection(bare)
    assert np.array_equal(p, O.graph_nested_dissection(A))
    assert _flops(A, p) < 0.05 * _flops(A, O.identity_ordering(A.n))


def test_best_nested_dissection_takes_the_one_with_fewer_flops():
    grid = M.grid_laplacian_3d(16, 2)                  # the pattern's ordering wins here
    vec = M.vector_laplacian_3d(10, 3)                 # the geometric one wins here
    for A in (grid, vec):
        best = O.best_nested_dissection(A)
        f = [_flops(A, O.nested_dissection(A)), _flops(A, O.graph_nested_dissection(A))]
        assert _flops(A, best) == min(f)
    assert np.array_equal(O.best_nested_dissection(grid), O.graph_nested_dissection(grid))
    assert np.array_equal(O.best_nested_dissection(vec), O.nested_dissection(vec))
