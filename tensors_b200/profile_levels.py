"""Per-level breakdown of one factorization and one 16-RHS solve (direct
launches timed by events).

    python -m tensors_b200.profile_levels [--grid 64]

Prints, for every level of the front tree, the milliseconds spent in each
launch kind, and writes the raw per-launch list as JSON to stdout's last line.
"""
from __future__ import annotations

import argparse
import collections
import json


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, default=64)
    args = ap.parse_args()
    import torch

    from tensors_b200 import build as tb_build
    from tensors_b200 import matrices, ordering
    from tensors_b200.cholesky import CholeskyDecomposition

    tb_build.build()
    A = matrices.grid_laplacian_3d(args.grid, 0x5EED0002, 1e-6)
    chol = CholeskyDecomposition(A.outer, A.inner, ordering.nested_dissection(A))
    vals = torch.tensor(A.values, device="cuda")
    chol.SetProfiling(True)
    for _ in range(3):
        assert chol.NumericFactorization(vals, 0.0) == 0
    prof = chol.LaunchProfile()
    per = collections.defaultdict(lambda: collections.defaultdict(float))
    cnt = collections.defaultdict(lambda: collections.defaultdict(int))
    for kind, level, step, tasks, ms in prof:
        per[level][kind] += ms
        cnt[level][kind] += 1
    kinds = ["assemble", "zero", "extend", "potrf", "trsm", "gemm", "invert"]
    print("level " + " ".join(f"{k:>14s}" for k in kinds) + "        total")
    for level in sorted(per):
        row = per[level]
        print(f"{level:5d} " + " ".join(f"{row[k]:8.3f}ms/{cnt[level][k]:4d}" for k in kinds) + f" {sum(row.values()):10.3f}")
    B = torch.randn(A.n, 16, dtype=torch.float64, device="cuda")
    X = torch.empty_like(B)
    for _ in range(3):
        chol.Solve(B, X)
    torch.cuda.synchronize()
    sprof = chol.SolveProfile()
    sper = collections.defaultdict(lambda: [0.0, 0, 0.0, 0, 0])
    for sweep, level, step, tasks, ms in sprof:
        e = sper[level]
        e[2 * sweep] += ms
        e[2 * sweep + 1] += 1
        e[4] = max(e[4], tasks)
    print("level  forward ms/launches   back ms/launches  max tasks")
    for level in sorted(sper):
        f, fc, b, bc, mt = sper[level]
        print(f"{level:5d} {f:10.3f}/{fc:4d}      {b:10.3f}/{bc:4d}   {mt:8d}")
    print(f"solve total {sum(x[4] for x in sprof):.3f} ms over {len(sprof)} launches")
    print(json.dumps({"factor": prof, "solve": sprof}))


if __name__ == "__main__":
    main()
