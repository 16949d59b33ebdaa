"""Generates the golden fixtures in this directory from the reference itself.

Each fixture holds a small SPD matrix, its fill-reducing permutation, and
everything the reference's own Sparse::CholeskyDecomposition (compiled from
its headers by oracle/Makefile into oracle/_ref) produces for it: the
symbolic arrays, the factor values in its layout, the return status, a
solve with three right-hand sides and the log-determinant.

Run from the repository root (needs the reference checkout, which only the
build container has):

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402
from tensors_b200 import matrices as M  # noqa: E402
from tensors_b200 import ordering as O  # noqa: E402


def tridiagonal(n):
    rows = np.concatenate([np.arange(n), np.arange(n - 1), np.arange(1, n)])
    cols = np.concatenate([np.arange(n), np.arange(1, n), np.arange(n - 1)])
    vals = np.concatenate([np.full(n, 2.0), np.full(n - 1, -1.0), np.full(n - 1, -1.0)])
    return M.from_coo(n, rows, cols, vals)


def arrow():
    outer = np.array([0, 2, 4, 7], dtype=np.int64)
    inner = np.array([0, 2, 1, 2, 0, 1, 2], dtype=np.int32)
    vals = np.array([-4.0, 1.0, 9.0, 1.0, 1.0, 1.0, 100.0])
    return M.CSRMatrix(n=3, outer=outer, inner=inner, values=vals)


def two_components():
    a = M.grid_laplacian_2d(5, 0.5)
    b = M.grid_laplacian_2d(4, 0.5)
    n = a.n + b.n
    ra = np.repeat(np.arange(a.n), np.diff(a.outer))
    rb = np.repeat(np.arange(b.n), np.diff(b.outer)) + a.n
    return M.from_coo(n, np.concatenate([ra, rb]), np.concatenate([a.inner, b.inner + a.n]),
                      np.concatenate([a.values, b.values]))


def cases():
    out = []
    A = M.grid_laplacian_2d(12, 0.0)
    for strat in ("maximal", "fundamental", "amalgamated"):
        out.append((f"grid2d12_nd_{strat}", A, O.nested_dissection(A, 8), strat, 1e-2))
    A = M.grid_laplacian_2d(10, 0.0)
    out.append(("grid2d10_random_maximal", A, np.random.default_rng(10).permutation(A.n).astype(np.int32), "maximal", 1e-2))
    A = M.grid_laplacian_3d(6, 0x5EED0002, 1e-2)
    out.append(("grid3d6_nd_maximal", A, O.nested_dissection(A, 8), "maximal", 0.0))
    A = M.vector_laplacian_3d(3, 0x5EED0003)
    out.append(("vector3d3_nd_maximal", A, O.nested_dissection(A, 4), "maximal", 1e-2))
    A = M.delaunay_laplacian(300, 0x5EED0004)
    out.append(("delaunay300_nd_fundamental", A, O.nested_dissection(A, 8), "fundamental", 1e-3))
    out.append(("tridiagonal50_identity_maximal", tridiagonal(50), None, "maximal", 0.0))
    out.append(("arrow3_identity_fundamental", arrow(), None, "fundamental", 0.0))
    A = two_components()
    out.append(("two_components_nd_maximal", A, np.random.default_rng(2).permutation(A.n).astype(np.int32), "maximal", 0.0))
    D = M.CSRMatrix(n=7, outer=np.arange(8, dtype=np.int64), inner=np.arange(7, dtype=np.int32),
                    values=np.array([4.0, -9.0, 1.0, 2.0, -1.0, 16.0, 3.0]))
    out.append(("diagonal7_identity_maximal", D, None, "maximal", 0.0))
    return out


def main():
    oracle.build(with_reference=True)
    for name, A, perm, strat, reg in cases():
        r = oracle.RefCholesky(A.n, A.outer, A.inner, perm, strat, threads=1)
        arrays = {k: r.array(k) for k in oracle.ARRAYS}
        status = r.factor(A.values, reg)
        tri, rec = r.factor_values()
        B = np.random.default_rng(A.n).standard_normal((A.n, 3))
        X = r.solve(B) if status == 0 else np.zeros_like(B)
        logdet = r.log_det() if status == 0 else np.nan
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"),
            n=A.n, outer=A.outer, inner=A.inner, values=A.values,
            perm=np.array([], dtype=np.int32) if perm is None else perm,
            has_perm=perm is not None, strategy=strat, reg=reg,
            status=status, tri=tri, rec=rec, B=B, X=X, logdet=logdet,
            **{f"arr_{k}": v for k, v in arrays.items()},
        )
        print(f"{name}: n={A.n} supernodes={r.sn_count()} status={status}")


if __name__ == "__main__":
    main()
