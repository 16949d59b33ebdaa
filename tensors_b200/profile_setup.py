"""Host set-up time of the Cholesky path (no GPU needed): fill-reducing
ordering (geometric, and from the pattern alone), symbolic analysis (eTree, postorder, supernodes, permuted pattern),
device-plan build, and the plan's bounds check, on the C2 and C3 workloads.

    python -m tensors_b200.profile_setup [--repeat 3]

Prints one line per workload with the median over the repeats.
"""
from __future__ import annotations

import argparse
import os
import statistics
import time


def _one(A, repeat):
    from tensors_b200 import ordering
    from tensors_b200.cholesky import CholeskyDecomposition

    rows = []
    for _ in range(repeat):
        t = time.perf_counter()
        ordering.graph_nested_dissection(A)
        t0 = time.perf_counter()
        perm = ordering.nested_dissection(A)
        t1 = time.perf_counter()
        c = CholeskyDecomposition(A.outer, A.inner, perm)
        c.SymbolicFactorization()
        st = c.PlanStats()
        t2 = time.perf_counter()
        c.CheckPlan()
        t3 = time.perf_counter()
        rows.append(((t1 - t0) * 1e3, st["analyze_us"] * 1e-3, st["plan_us"] * 1e-3, (t3 - t2) * 1e3,
                     (t2 - t1) * 1e3, (t0 - t) * 1e3))
    return [statistics.median(col) for col in zip(*rows)], st


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--repeat", type=int, default=3)
    args = ap.parse_args()
    from tensors_b200 import build as tb_build
    from tensors_b200 import matrices

    tb_build.build()
    cases = [("C2 64^3 7-point", matrices.grid_laplacian_3d(64, 0x5EED0002, 1e-6)),
             ("C3 48^3 3-dof 27-point", matrices.vector_laplacian_3d(48, 0x5EED0003, 1e-2))]
    print(f"host threads: {os.cpu_count()}")
    for name, A in cases:
        (nd, an, pl, ck, total, gnd), st = _one(A, args.repeat)
        print(f"{name}: n {A.n}, nnz {A.nnz}, fronts {st['fronts']}, GEMM tasks {st['gemm_tasks']}: "
              f"geometric ordering {nd:.0f} ms (pattern-only ordering {gnd:.0f} ms), analysis {an:.0f} ms, "
              f"plan {pl:.0f} ms, plan check {ck:.0f} ms (symbolic call {total:.0f} ms)")


if __name__ == "__main__":
    main()
