"""Synthetic SPD test matrices in the CSR form the Cholesky path consumes.

Every generator returns a :class:`CSRMatrix` holding the *full* symmetric
pattern with a structurally present diagonal and sorted column indices, the
input contract of ``Sparse::CholeskyDecomposition``
(src/Sparse/CholeskyDecomposition.hpp:63-65, :404-423), plus the node
coordinates that the geometric nested-dissection orderings use.

Random inputs use ``numpy.random.Generator(PCG64(seed))`` so that a seed
fixes every value on every host.  The workloads:

* :func:`grid_laplacian_2d` -- the reference's own test matrix
  ``Sparse::GridLaplacian`` (src/Sparse/GridLaplacian.hpp:11-77): 5-point graph
  Laplacian of a ``g x g`` grid plus ``mass * I``.
* :func:`grid_laplacian_3d` -- 7-point graph Laplacian of a ``g^3`` grid with
  per-edge conductivities ``exp(N(0,1))`` plus a diagonal shift.
* :func:`vector_laplacian_3d` -- 3 degrees of freedom per node, 27-point
  stencil, SPD 3x3 edge blocks ``B = G G^T + 0.1 I`` with ``G`` i.i.d. N(0,1);
  ``A = sum_e [[B,-B],[-B,B]]`` (positive semidefinite: constant fields span
  its null space, so a diagonal shift is passed to the factorization).
* :func:`delaunay_laplacian` -- cotangent Laplacian of the Delaunay
  triangulation of ``m`` uniform points in the unit square plus ``shift``
  times the lumped (one third of incident triangle areas) mass matrix.
* :func:`mesh_laplacian` -- the same operator on a jittered-grid point set.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

__all__ = [
    "CSRMatrix",
    "from_coo",
    "grid_laplacian_2d",
    "grid_laplacian_3d",
    "vector_laplacian_3d",
    "delaunay_laplacian",
    "mesh_laplacian",
    "csr_matvec",
]


@dataclass
class CSRMatrix:
    """Square CSR matrix with int64 row pointers and int32 column indices."""

    n: int
    outer: np.ndarray          # int64, n + 1
    inner: np.ndarray          # int32, nnz
    values: np.ndarray         # float64, nnz
    coords: np.ndarray | None = None   # node coordinates (nodes x dim)
    dofs_per_node: int = 1
    meta: dict = field(default_factory=dict)

    @property
    def nnz(self) -> int:
        return int(self.outer[-1])

    def to_scipy(self):
        import scipy.sparse as sp

        return sp.csr_matrix((self.values, self.inner, self.outer), shape=(self.n, self.n))

    def diagonal(self) -> np.ndarray:
        rows = np.repeat(np.arange(self.n, dtype=np.int64), np.diff(self.outer))
        d = np.zeros(self.n)
        mask = rows == self.inner
        d[rows[mask]] = self.values[mask]
        return d


def from_coo(n: int, rows: np.ndarray, cols: np.ndarray, vals: np.ndarray, **kw) -> CSRMatrix:
    """Sum duplicate (row, col) triples into a sorted CSR matrix."""
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    vals = np.asarray(vals, dtype=np.float64)
    key = rows * n + cols
    order = np.argsort(key, kind="stable")
    key = key[order]
    vals = vals[order]
    uniq, start = np.unique(key, return_index=True)
    summed = np.add.reduceat(vals, start) if len(vals) else vals
    r = (uniq // n).astype(np.int64)
    c = (uniq % n).astype(np.int32)
    outer = np.zeros(n + 1, dtype=np.int64)
    np.add.at(outer, r + 1, 1)
    outer = np.cumsum(outer)
    return CSRMatrix(n=n, outer=outer, inner=np.ascontiguousarray(c),
                     values=np.ascontiguousarray(summed), **kw)


def _edge_laplacian(n: int, a: np.ndarray, b: np.ndarray, w: np.ndarray, diag_extra: np.ndarray, **kw) -> CSRMatrix:
    rows = np.concatenate([a, b, a, b, np.arange(n)])
    cols = np.concatenate([b, a, a, b, np.arange(n)])
    vals = np.concatenate([-w, -w, w, w, diag_extra])
    return from_coo(n, rows, cols, vals, **kw)


def grid_laplacian_2d(g: int, mass: float = 1.0) -> CSRMatrix:
    """``Sparse::GridLaplacian(g, mass)``: 5-point graph Laplacian + mass*I."""
    idx = np.arange(g * g, dtype=np.int64).reshape(g, g)
    a = np.concatenate([idx[:, :-1].ravel(), idx[:-1, :].ravel()])
    b = np.concatenate([idx[:, 1:].ravel(), idx[1:, :].ravel()])
    w = np.ones(len(a))
    n = g * g
    yy, xx = np.meshgrid(np.arange(g), np.arange(g), indexing="ij")
    coords = np.stack([yy.ravel(), xx.ravel()], axis=1).astype(np.float64)
    return _edge_laplacian(n, a, b, w, np.full(n, float(mass)), coords=coords,
                           meta={"kind": "grid2d", "grid": g, "mass": mass})


def grid_laplacian_3d(g: int, seed: int, shift: float = 1e-6) -> CSRMatrix:
    """7-point Laplacian on ``g^3`` with lognormal(0,1) edge weights + shift*I."""
    rng = np.random.Generator(np.random.PCG64(seed))
    idx = np.arange(g ** 3, dtype=np.int64).reshape(g, g, g)
    a = np.concatenate([idx[:-1, :, :].ravel(), idx[:, :-1, :].ravel(), idx[:, :, :-1].ravel()])
    b = np.concatenate([idx[1:, :, :].ravel(), idx[:, 1:, :].ravel(), idx[:, :, 1:].ravel()])
    w = np.exp(rng.standard_normal(len(a)))
    n = g ** 3
    zz, yy, xx = np.meshgrid(np.arange(g), np.arange(g), np.arange(g), indexing="ij")
    coords = np.stack([zz.ravel(), yy.ravel(), xx.ravel()], axis=1).astype(np.float64)
    return _edge_laplacian(n, a, b, w, np.full(n, float(shift)), coords=coords,
                           meta={"kind": "grid3d", "grid": g, "seed": seed, "shift": shift})


def vector_laplacian_3d(g: int, seed: int, shift: float = 0.0) -> CSRMatrix:
    """3-dof, 27-point vector Laplacian with SPD 3x3 edge blocks (+ shift*I)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    idx = np.arange(g ** 3, dtype=np.int64).reshape(g, g, g)
    a_list, b_list = [], []
    # the 13 "forward" neighbour offsets of the 26-neighbourhood
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                if (dz, dy, dx) <= (0, 0, 0):
                    continue
                sz = slice(max(0, -dz), g - max(0, dz))
                sy = slice(max(0, -dy), g - max(0, dy))
                sx = slice(max(0, -dx), g - max(0, dx))
                tz = slice(max(0, dz), g - max(0, -dz))
                ty = slice(max(0, dy), g - max(0, -dy))
                tx = slice(max(0, dx), g - max(0, -dx))
                a_list.append(idx[sz, sy, sx].ravel())
                b_list.append(idx[tz, ty, tx].ravel())
    a = np.concatenate(a_list)
    b = np.concatenate(b_list)
    ne = len(a)
    G = rng.standard_normal((ne, 3, 3))
    B = G @ np.transpose(G, (0, 2, 1)) + 0.1 * np.eye(3)
    nodes = g ** 3
    n = 3 * nodes
    r3 = np.arange(3)
    # block (p,q) entries: rows 3p+i, cols 3q+j
    ii = np.broadcast_to(r3[None, :, None], (ne, 3, 3))
    jj = np.broadcast_to(r3[None, None, :], (ne, 3, 3))
    ap = a[:, None, None] * 3
    bp = b[:, None, None] * 3
    rows = np.concatenate([(ap + ii).ravel(), (bp + ii).ravel(), (ap + ii).ravel(), (bp + ii).ravel()])
    cols = np.concatenate([(ap + jj).ravel(), (bp + jj).ravel(), (bp + jj).ravel(), (ap + jj).ravel()])
    vals = np.concatenate([B.ravel(), B.ravel(), -B.ravel(), -B.ravel()])
    if shift != 0.0:
        rows = np.concatenate([rows, np.arange(n)])
        cols = np.concatenate([cols, np.arange(n)])
        vals = np.concatenate([vals, np.full(n, float(shift))])
    zz, yy, xx = np.meshgrid(np.arange(g), np.arange(g), np.arange(g), indexing="ij")
    coords = np.stack([zz.ravel(), yy.ravel(), xx.ravel()], axis=1).astype(np.float64)
    return from_coo(n, rows, cols, vals, coords=coords, dofs_per_node=3,
                    meta={"kind": "vector3d", "grid": g, "seed": seed, "shift": shift})


def delaunay_laplacian(m: int, seed: int, shift: float = 1e-3) -> CSRMatrix:
    """Cotangent Laplacian of a random Delaunay mesh + shift * lumped mass."""
    from scipy.spatial import Delaunay

    rng = np.random.Generator(np.random.PCG64(seed))
    pts = rng.random((m, 2))
    tri = Delaunay(pts).simplices.astype(np.int64)
    return _cotangent_laplacian(pts, tri, shift, {"kind": "delaunay", "m": m, "seed": seed, "shift": shift})


def _cotangent_laplacian(pts, tri, shift, meta, relative: bool = False) -> CSRMatrix:
    m = len(pts)
    P = pts[tri]                                  # (t, 3, 2)
    rows, cols, vals = [], [], []
    for k in range(3):
        i, j, o = (k + 1) % 3, (k + 2) % 3, k     # edge (i,j) opposite vertex o
        u = P[:, i] - P[:, o]
        v = P[:, j] - P[:, o]
        cross = np.abs(u[:, 0] * v[:, 1] - u[:, 1] * v[:, 0])
        cot = (u * v).sum(1) / np.maximum(cross, 1e-300)
        w = 0.5 * cot
        a, b = tri[:, i], tri[:, j]
        rows += [a, b, a, b]
        cols += [b, a, a, b]
        vals += [-w, -w, w, w]
    e1 = P[:, 1] - P[:, 0]
    e2 = P[:, 2] - P[:, 0]
    area = 0.5 * np.abs(e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0])
    mass = np.zeros(m)
    for k in range(3):
        np.add.at(mass, tri[:, k], area / 3.0)
    rows.append(np.arange(m))
    cols.append(np.arange(m))
    vals.append(shift * mass / (mass.mean() if relative else 1.0))
    return from_coo(m, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals), coords=pts, meta=meta)


def mesh_laplacian(m: int, seed: int, shift: float = 1e-3, relative: bool = False) -> CSRMatrix:
    """Cotangent Laplacian + shift * lumped mass of a quality 2D mesh: the Delaunay
    triangulation of about m points on a jittered grid (every point moved by up to
    a quarter cell), which keeps the angles bounded away from 0 and pi -- unlike
    uniform random points, whose hull slivers give cotangent weights of ~1e6.
    relative: the lumped mass is scaled to mean 1, so the diagonal shift averages
    `shift` at any resolution (an absolute shift times a mass of ~1/m makes kappa
    grow like m / shift)."""
    from scipy.spatial import Delaunay

    rng = np.random.Generator(np.random.PCG64(seed))
    g = max(2, int(round(np.sqrt(m))))
    h = 1.0 / (g - 1)
    yy, xx = np.meshgrid(np.arange(g) * h, np.arange(g) * h, indexing="ij")
    pts = np.stack([xx.ravel(), yy.ravel()], 1) + rng.uniform(-0.25 * h, 0.25 * h, size=(g * g, 2))
    tri = Delaunay(pts).simplices.astype(np.int64)
    return _cotangent_laplacian(pts, tri, shift, {"kind": "mesh", "m": g * g, "seed": seed, "shift": shift,
                                                  "relative": relative}, relative)


def csr_matvec(A: CSRMatrix, X: np.ndarray) -> np.ndarray:
    """A @ X for a row-major n x k (or length-n) array, in float64."""
    return A.to_scipy() @ X
