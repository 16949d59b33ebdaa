"""Nested-dissection ordering: validity and fill reduction."""
from __future__ import annotations

import numpy as np

from tensors_b200 import matrices as M
from tensors_b200 import ordering as O
from tensors_b200.cholesky import CholeskyDecomposition


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
