"""Fill-reducing orderings for the Cholesky path.

The reference takes its fill-reducing permutation from METIS or SuiteSparse
AMD (src/Sparse/Metis.hpp:81, src/Sparse/ApproximateMinimumDegree.hpp:58),
neither of which is available here, so this module supplies a project-written
geometric nested dissection: recursively split the node set at the median of
its longest coordinate axis, take the nodes of the lower half that touch the
upper half as the vertex separator, order both halves recursively and the
separator last.  For stencil matrices on grids the separator is one grid
plane, which is the classical nested-dissection ordering.

The returned array follows the reference's constructor convention
(CholeskyDecomposition.hpp:336-345, ``Inverse::False``): ``perm[i]`` is the
original index placed at position ``i``.
"""
from __future__ import annotations

import numpy as np

from .matrices import CSRMatrix

__all__ = ["nested_dissection", "graph_nested_dissection", "best_nested_dissection", "identity_ordering",
           "is_permutation"]


def is_permutation(p: np.ndarray, n: int) -> bool:
    p = np.asarray(p)
    if p.shape != (n,):
        return False
    seen = np.zeros(n, dtype=bool)
    if n and (p.min() < 0 or p.max() >= n):
        return False
    seen[p] = True
    return bool(seen.all())


def identity_ordering(n: int) -> np.ndarray:
    return np.arange(n, dtype=np.int32)


def _node_graph(A: CSRMatrix):
    """CSR adjacency between nodes (dofs of one node collapsed)."""
    d = A.dofs_per_node
    if d == 1:
        return A.outer, A.inner.astype(np.int64), A.n
    import scipy.sparse as sp

    nodes = A.n // d
    rows = np.repeat(np.arange(A.n, dtype=np.int64), np.diff(A.outer)) // d
    cols = A.inner.astype(np.int64) // d
    G = sp.csr_matrix((np.ones(len(rows), dtype=np.int8), (rows, cols)), shape=(nodes, nodes))
    G.sum_duplicates()
    return G.indptr.astype(np.int64), G.indices.astype(np.int64), nodes


def graph_nested_dissection(A: CSRMatrix, leaf_size: int = 64, thread_count: int = 0) -> np.ndarray:
    """Nested dissection from the pattern alone (native ``tb_nested_dissection``): George's
    automatic nested dissection with rooted level structures from pseudo-peripheral nodes.
    Needs no coordinates, so it orders any matrix (one read from a file, say); the dofs of a
    node (``A.dofs_per_node`` consecutive rows) stay together.  ``thread_count`` <= 0: all host
    threads; the order is the same for every thread count."""
    from ._lib import lib
    from .cholesky import _check

    outer = np.ascontiguousarray(A.outer, dtype=np.int64)
    inner = np.ascontiguousarray(A.inner, dtype=np.int32)
    perm = np.zeros(A.n, dtype=np.int32)
    _check(lib().tb_nested_dissection(int(A.n), outer.ctypes.data, inner.ctypes.data, int(A.dofs_per_node),
                                      int(leaf_size), int(thread_count), perm.ctypes.data))
    return perm


def nested_dissection(A: CSRMatrix, leaf_size: int = 64) -> np.ndarray:
    """Geometric nested dissection of ``A`` using ``A.coords`` (see module doc); a matrix without
    coordinates is ordered by :func:`graph_nested_dissection`."""
    if A.coords is None:
        return graph_nested_dissection(A, leaf_size)
    indptr, indices, nodes = _node_graph(A)
    coords = np.asarray(A.coords, dtype=np.float64)
    if coords.shape[0] != nodes:
        raise ValueError("coords must have one row per node")
    mark = np.zeros(nodes, dtype=bool)
    out: list[np.ndarray] = []

    def touches(group: np.ndarray, other: np.ndarray) -> np.ndarray:
        """Boolean mask: which nodes of `group` have a neighbour in `other`."""
        mark[other] = True
        starts = indptr[group]
        counts = indptr[group + 1] - starts
        if counts.sum() == 0:
            mark[other] = False
            return np.zeros(len(group), dtype=bool)
        pos = np.repeat(starts - np.concatenate([[0], np.cumsum(counts)[:-1]]), counts) + np.arange(counts.sum())
        hit = mark[indices[pos]].astype(np.int64)
        mark[other] = False
        csum = np.concatenate([[0], np.cumsum(hit)])
        ends = np.cumsum(counts)
        begins = ends - counts
        return (csum[ends] - csum[begins]) > 0

    # explicit stack of (node set, phase): phase 0 = split, 1 = emit separator
    stack: list[tuple[np.ndarray, int]] = [(np.arange(nodes, dtype=np.int64), 0)]
    while stack:
        group, phase = stack.pop()
        if phase == 1:
            out.append(group)
            continue
        if len(group) <= leaf_size:
            out.append(group)
            continue
        c = coords[group]
        ext = c.max(axis=0) - c.min(axis=0)
        axis = int(np.argmax(ext))
        x = c[:, axis]
        s = np.median(x)
        lower = x < s
        if lower.sum() == 0 or lower.sum() == len(group):
            lower = x <= s
            if lower.sum() == 0 or lower.sum() == len(group):
                out.append(group)
                continue
        left, right = group[lower], group[~lower]
        sep_mask = touches(left, right)
        sep = left[sep_mask]
        left = left[~sep_mask]
        # postorder: left, right, then separator (stack is LIFO)
        stack.append((sep, 1))
        stack.append((right, 0))
        stack.append((left, 0))
    node_order = np.concatenate(out) if out else np.zeros(0, dtype=np.int64)
    d = A.dofs_per_node
    if d > 1:
        node_order = (node_order[:, None] * d + np.arange(d)[None, :]).ravel()
    return node_order.astype(np.int32)


def best_nested_dissection(A: CSRMatrix, leaf_size: int = 64) -> np.ndarray:
    """The geometric dissection (when ``A`` has coordinates) or the one from the pattern alone,
    whichever gives fewer factor flops by the symbolic analysis (host only, one analysis each).
    Neither wins everywhere: on 7-point grids the pattern's level structures cut diagonally and
    need about half the flops; on 27-point stencils the grid planes need about a third."""
    from .cholesky import CholeskyDecomposition

    candidates = [graph_nested_dissection(A, leaf_size)]
    if A.coords is not None:
        candidates.insert(0, nested_dissection(A, leaf_size))
    flops = [CholeskyDecomposition(A.outer, A.inner, p).FlopCount()[0] for p in candidates]
    return candidates[int(np.argmin(flops))]
