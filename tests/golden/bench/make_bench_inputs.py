"""Writes the fill-reducing permutation of the FP64 benchmark's matrix.

The benchmark factors the 7-point Laplacian of a 64^3 grid (n = 262,144,
lognormal(0,1) edge conductivities from seed 0x5EED0002, shift 1e-6) under the
nested dissection with fewer factor flops, which on this grid is the one from
the pattern alone (tb_nested_dissection, about half the flops of the geometric
one).  The reference has no ordering of its own here (its METIS and AMD
wrappers need libraries that are absent), so both benchmark arms take this
permutation as input.  The reference arm reads it from this file, so that it
runs the reference's own code without loading this library;
tests/test_bench_inputs.py checks that the file still equals what the library
computes.

    python tests/golden/bench/make_bench_inputs.py

Output: tests/golden/bench/c2_grid64_graph_nd.npz, the permutation delta-encoded
(perm = cumsum(delta)) to keep the file small.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(os.path.dirname(HERE)))
OUT = os.path.join(HERE, "c2_grid64_graph_nd.npz")
GRID, SEED, SHIFT = 64, 0x5EED0002, 1e-6


def compute() -> np.ndarray:
    sys.path.insert(0, ROOT)
    from tensors_b200 import matrices, ordering

    A = matrices.grid_laplacian_3d(GRID, SEED, SHIFT)
    return ordering.graph_nested_dissection(A)


def load(path: str = OUT) -> np.ndarray:
    z = np.load(path)
    return np.cumsum(z["delta"].astype(np.int64)).astype(np.int32)


if __name__ == "__main__":
    perm = compute()
    delta = np.diff(perm.astype(np.int64), prepend=0).astype(np.int32)
    np.savez_compressed(OUT, delta=delta, grid=GRID, seed=SEED, shift=SHIFT)
    assert np.array_equal(load(OUT), perm)
    print(f"wrote {OUT}: n={len(perm)}")
