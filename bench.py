#!/usr/bin/env python3
"""Benchmark: supernodal Cholesky factor + solve on one or more B200s.

Workload (one step): NumericFactorization + Solve with 16 right-hand sides of
the 7-point Laplacian of a 64^3 grid (n = 262,144) with per-edge
conductivities exp(N(0,1)) and a 1e-6 diagonal shift, plain FP64, under the
nested dissection with fewer factor flops (on this grid the one from the
pattern alone: about half the flops of the geometric one).  Inputs are seeded
synthetic data (no dataset exists for this path).  Symbolic analysis is done
once before timing, as in the reference's driver
(Example_SparseCholesky/main.cpp:135 vs :147).

The metric is factor+solve throughput in GFLOP/s, counting the reference's
algorithmic flops once: factor Sum_s [n0^3/3 + n0^2 n1 + n0 n1^2] over the
reference's supernodes plus solve 4 k nnz(U); ms_per_step is the factor+solve
time.  Every run checks the relative residual ||B - A X|| / ||B|| on the
device; the CPU-baseline leg also runs the reference's own code on the same
system and reports the forward difference of the two solutions.

The default line also carries the mixed-precision comparison on the 3-dof
27-point vector Laplacian of a 48^3 grid (FP32 factor with 3xTF32 tensor-core
updates + FP64 refinement vs plain FP64, both to 1e-12): `config.mixed_vs_fp64`.

Multi-GPU (torchrun): the workload is replicated -- each rank factors and
solves its own system (weak scaling, no collective on the data path).

`--impl reference` times the reference's own CPU implementation (compiled
from its headers into oracle/_ref) on all host cores for the same metric on
the same system: each step is one full factor + solve.  It takes the
permutation from tests/golden/bench/c2_grid64_graph_nd.npz, so that process loads
only the reference's library.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

GRID = 64
SEED = 0x5EED0002
SHIFT = 1e-6
NRHS = 16
L2_FLUSH_BYTES = 256 << 20
# The permutation of the 64^3 system under the pattern-only nested dissection,
# written by tests/golden/bench/make_bench_inputs.py (checked against the library by
# tests/test_bench_inputs.py): the reference arm reads it instead of running
# this library's ordering.
PERM_FIXTURE = os.path.join(ROOT, "tests", "golden", "bench", "c2_grid64_graph_nd.npz")

# The system's nested dissection: "graph" (from the pattern alone, the default:
# the fewer-flop ordering on this grid) or "geometric" (grid planes from the
# node coordinates, twice the factor flops here).
ORDERING = "graph"
METRIC = "factor+solve GFLOP/s (FP64, 64^3 7-pt Laplacian, 16 RHS)"


def c2_permutation(A, name, product=True):
    """Fill-reducing order of the benchmark matrix.  product=False (reference arm): the geometric
    order is pure numpy and the pattern-only order of the 64^3 system comes from the fixture."""
    from tensors_b200 import ordering

    if name == "geometric":
        return ordering.nested_dissection(A)
    if not product and A.n == 64 ** 3 and os.path.exists(PERM_FIXTURE):
        z = np.load(PERM_FIXTURE)
        return np.cumsum(z["delta"].astype(np.int64)).astype(np.int32)
    return ordering.graph_nested_dissection(A)


def build_problem(grid: int | None = None, ordering_name: str | None = None, product: bool = True):
    grid = GRID if grid is None else grid
    from tensors_b200 import matrices

    A = matrices.grid_laplacian_3d(grid, SEED, SHIFT)
    perm = c2_permutation(A, ORDERING if ordering_name is None else ordering_name, product)
    B = np.random.default_rng(SEED + 1).standard_normal((A.n, NRHS))
    return A, perm, B


def config_dict(extra=None):
    c = {
        "workload": f"3D 7-point Laplacian {GRID}^3 (n={GRID**3}), lognormal(0,1) edge conductivities, "
                    f"shift {SHIFT:g}, nested dissection, {NRHS} RHS N(0,1), FP64 factor+solve",
        "grid": GRID, "n": GRID ** 3, "nrhs": NRHS, "seed": SEED,
        "supernode_strategy": "Maximal",
        "ordering": ("nested dissection from the pattern alone (fewer factor flops than the geometric one)"
                     if ORDERING == "graph" else "geometric nested dissection"),
        "l2": "256 MiB buffer written between timed steps (inputs and factor also exceed L2)",
    }
    if extra:
        c.update(extra)
    return c


class ClockSampler:
    """Samples nvidia-smi clocks / throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measure_dgemm_tflops(torch, dev):
    """cuBLAS FP64 GEMM throughput (the FP64 tensor-core reference denominator)."""
    n = 8192
    a = torch.randn(n, n, device=dev, dtype=torch.float64)
    b = torch.randn(n, n, device=dev, dtype=torch.float64)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize(dev)
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = max(best, 2.0 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    return best


def reference_run(A, perm, B, threads, steps=1, warmup=0):
    """Times the reference's own CPU factor+solve (oracle/_ref) on this host: `threads` tree threads, one
    BLAS thread each (the reference parallelises over the assembly tree).  Its flops come from its own
    supernodes, so this needs nothing from this library."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    if not oracle.ref_available():
        return None
    ref = oracle.RefCholesky(A.n, A.outer, A.inner, perm, "maximal", threads=threads, blas_threads=1)
    ref.symbolic()
    n0 = np.diff(ref.array("SN_rp")).astype(np.float64)
    n1 = np.diff(ref.array("SN_outer")).astype(np.float64)
    factor_flops = float((n0 ** 3 / 3.0 + n0 ** 2 * n1 + n0 * n1 ** 2).sum())
    nnz_u = float((n0 * (n0 + 1.0) / 2.0 + n0 * n1).sum())
    k = 1 if B.ndim == 1 else B.shape[1]
    times = []
    X = None
    st = 0
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        st = ref.factor(A.values, 0.0)
        X = ref.solve(B, parallel=False)
        dt = time.perf_counter() - t0
        if i >= warmup:
            times.append(dt)
    res = np.linalg.norm(B - A.to_scipy() @ X) / np.linalg.norm(B)
    return {"seconds": times, "status": st, "relres": float(res), "X": X,
            "factor_flops": factor_flops, "nnz_u": nnz_u, "flops": factor_flops + 4.0 * k * nnz_u}


def run_reference(args):
    """The reference arm: the reference's own CPU code on the benchmark's system, every host thread."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    A, perm, B = build_problem(args.grid, product=False)
    threads = os.cpu_count() or 1
    r = reference_run(A, perm, B, threads, steps=args.steps, warmup=args.warmup)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libtb_ref.so not built (needs the reference checkout)"}))
        return 0
    t = statistics.mean(r["seconds"])
    v = r["flops"] / t / 1e9
    sample = f"one full factor + solve of the benchmark system per step ({threads} tree threads, 1 BLAS thread each)"
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": v, "unit": "GFLOP/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded)",
        "config": config_dict({"relres": r["relres"], "cpu_threads": threads, "factor_gflop": r["factor_flops"] / 1e9,
                               "seconds": r["seconds"]}),
        "cpu_baseline": {"value": v, "unit": "GFLOP/s", "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_for_profiler(args):
    """The plain workload for ncu: (warmup + steps) x (factor + solve), direct launches; the
    headline Laplacian, or with --workload c3 the vector Laplacian (--grid: its edge)."""
    import torch
    from tensors_b200 import build as tb_build
    from tensors_b200.cholesky import CholeskyDecomposition

    tb_build.build()
    if args.workload == "c3":
        from tensors_b200 import matrices, ordering

        A = matrices.vector_laplacian_3d(args.grid or C3_GRID, C3_SEED, C3_SHIFT)
        perm = ordering.nested_dissection(A)
        B_host = np.random.default_rng(C3_SEED + 1).standard_normal((A.n, C3_NRHS))
    else:
        A, perm, B_host = build_problem(args.grid)
    chol = CholeskyDecomposition(A.outer, A.inner, perm)
    chol.SetPrecision(args.precision)
    chol.SymbolicFactorization()
    chol.SetUseGraph(False)
    vals = torch.tensor(A.values, device="cuda")
    B = torch.tensor(B_host, device="cuda")
    X = torch.empty_like(B)
    for _ in range(args.warmup + args.steps):
        assert chol.NumericFactorization(vals, 0.0) == 0
        chol.Solve(B, X)
    torch.cuda.synchronize()
    R = chol.Residual(B, X)
    torch.cuda.synchronize()
    print(json.dumps({"workload": args.workload or "c2", "grid": args.grid, "precision": args.precision,
                      "relres": float(torch.linalg.norm(R) / torch.linalg.norm(B)),
                      "launches": chol.LaunchCounts(), "plan": chol.PlanStats()}))
    return 0


# ------------------------------------------------------------ other configs
C3_GRID, C3_SEED, C3_SHIFT, C3_NRHS, C3_TARGET = 48, 0x5EED0003, 1e-2, 8, 1e-12
C3_NORTH_STAR_TARGET = 1e-10     # the mixed-vs-FP64 target of the path's goal (the configuration says 1e-12)
C4_COUNT, C4_SEED, C4_MIN, C4_MAX = 2000, 0x5EED0004, 500, 20000
# The random Delaunay meshes carry near-flat hull triangles whose cotangent
# weights reach ~1e6 while the lumped mass is ~1e-8: kappa ~1e12-1e14.  A plain
# FP64 direct solve attains a relative residual of only ~2e-8 on them, so the
# batch's refinement target is max(1e-10, 2 x what the reference's own FP64
# code attains on the same systems).
TARGET_RELRES = 1e-10


def _time_steps(torch, stream, fn, steps, warmup, barrier=None):
    """(mean ms of fn() per step, mean ms of its first phase) with CUDA events on `stream`;
    `barrier` (several ranks) lines the ranks up after the warm-up."""
    for _ in range(warmup):
        fn(None)
    torch.cuda.synchronize()
    if barrier is not None:
        barrier()
        torch.cuda.synchronize()
    tot, first = [], []
    for _ in range(steps):
        s, m, e = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        s.record(stream)
        fn(m)
        e.record(stream)
        e.synchronize()
        tot.append(s.elapsed_time(e))
        first.append(s.elapsed_time(m))
    return statistics.mean(tot), statistics.mean(first)


def c3_compare(torch, dev, steps, warmup, autotune=True):
    """Mixed precision vs FP64 on the 3-dof 27-point vector Laplacian (48^3 nodes, n = 331,776), 8 RHS.

    The stiffness sum_e [[B,-B],[-B,B]] with SPD edge blocks B = G G^T + 0.1 I is
    singular (rigid translations are in its null space), so the matrix carries
    a 1e-2 diagonal shift.  Both paths solve to the configuration's 1e-12
    relative residual target (the mixed path also to 1e-10, the target of the
    path's 2x goal); the FP64 path reaches ~1e-14 directly.  Returns per
    precision the step, factor and solve times, the relative residual and the
    refinement, plus the speed-up and the forward difference of the mixed
    solution from the FP64 one.
    """
    from tensors_b200 import build as tb_build
    from tensors_b200 import matrices, ordering
    from tensors_b200.cholesky import CholeskyDecomposition

    tb_build.build()
    A = matrices.vector_laplacian_3d(C3_GRID, C3_SEED, C3_SHIFT)
    perm = ordering.nested_dissection(A)
    B = torch.tensor(np.random.default_rng(C3_SEED + 1).standard_normal((A.n, C3_NRHS)), device=dev)
    vals = torch.tensor(A.values, device=dev)
    stream = torch.cuda.Stream(dev)
    prev = torch.cuda.current_stream(dev)
    torch.cuda.set_stream(stream)
    out, sols = {}, {}
    F = nnz_u = 0.0
    for prec in ("fp64", "mixed"):
        c = CholeskyDecomposition(A.outer, A.inner, perm)
        c.SetPrecision(prec)
        c.SetRefinement(C3_TARGET, 30)
        c.SetStream(stream)
        c.SymbolicFactorization()
        X = torch.empty_like(B)
        tuned = None
        if autotune:
            assert c.NumericFactorization(vals, 0.0) == 0
            tuned = c.AutotunePlan()["choice"]

        def step(mid):
            assert c.NumericFactorization(vals, 0.0) == 0
            if mid is not None:
                mid.record(stream)
            c.Solve(B, X)

        # the mixed path also to the north star's 1e-10 (the FP64 path reaches ~1e-14 either way)
        for target in ((C3_TARGET, C3_NORTH_STAR_TARGET) if prec == "mixed" else (C3_TARGET,)):
            c.SetRefinement(target, 30)
            with ClockSampler(dev.index or 0) as clocks:
                t, tf = _time_steps(torch, stream, step, steps, warmup)
            R = c.Residual(B, X)
            stream.synchronize()
            rr = float((torch.linalg.norm(R, dim=0) / torch.linalg.norm(B, dim=0)).max())
            F, nnz_u = c.FlopCount()
            key = prec if target == C3_TARGET else f"{prec}_{target:g}"
            out[key] = {"ms": t, "factor_ms": tf, "solve_ms": t - tf, "relres": rr, "target": target,
                        "plan_options": tuned, "refinement": c.RefinementInfo() if prec == "mixed" else None,
                        "precision_in_use": list(c.PrecisionInUse()), "clocks": clocks.summary()}
            if target == C3_TARGET:
                sols[prec] = X.clone()
        del c
    torch.cuda.set_stream(prev)
    flops = F + 4.0 * C3_NRHS * nnz_u
    return {"workload": f"3-dof 27-point vector Laplacian {C3_GRID}^3 (n={A.n}), SPD 3x3 edge blocks "
                        f"G G^T + 0.1 I, shift {C3_SHIFT:g}, geometric nested dissection, {C3_NRHS} RHS, "
                        f"target relres {C3_TARGET:g}",
            "factor_gflop": F / 1e9, "flops": flops, "fp64": out["fp64"], "mixed": out["mixed"],
            f"mixed_{C3_NORTH_STAR_TARGET:g}": out[f"mixed_{C3_NORTH_STAR_TARGET:g}"],
            "speedup_mixed_over_fp64": out["fp64"]["ms"] / out["mixed"]["ms"],
            f"speedup_mixed_over_fp64_at_{C3_NORTH_STAR_TARGET:g}": out["fp64"]["ms"] / out[f"mixed_{C3_NORTH_STAR_TARGET:g}"]["ms"],
            "forward_diff_mixed_vs_fp64": float(torch.linalg.norm(sols["mixed"] - sols["fp64"])
                                                / torch.linalg.norm(sols["fp64"])),
            "l2": "factor and matrix exceed L2"}


def run_c3(args):
    """The mixed-precision vs FP64 comparison (c3_compare) as its own line: GFLOP/s of the mixed path."""
    import torch

    dev = torch.device("cuda", 0)
    r = c3_compare(torch, dev, args.steps, args.warmup, not args.no_autotune)
    line = {
        "metric": "factor+solve GFLOP/s to 1e-12 relative residual, mixed precision (FP32 factor, 3xTF32 updates, "
                  "FP64 refinement) vs plain FP64, 48^3 3-dof 27-pt vector Laplacian, 8 RHS",
        "value": r["flops"] / (r["mixed"]["ms"] * 1e-3) / 1e9, "unit": "GFLOP/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["mixed"]["ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded)",
        "config": r,
    }
    print(json.dumps(line))
    return 0


def _c4_system(args):
    s, m = args
    from tensors_b200 import matrices, ordering

    A = matrices.delaunay_laplacian(int(m), C4_SEED + s, 1e-3)
    return A.outer, A.inner, A.values, ordering.nested_dissection(A)


def c4_sizes(count=C4_COUNT):
    """Point counts m ~ U[500, 20000] of the batch's meshes (system s has seed C4_SEED + s)."""
    return np.random.default_rng(C4_SEED).integers(C4_MIN, C4_MAX + 1, size=count)


def c4_systems(count=C4_COUNT, which=None):
    """The batch (or the systems `which` of it): Delaunay meshes of m ~ U[500, 20000] uniform points,
    cotangent Laplacian + 1e-3 lumped mass."""
    import multiprocessing as mp

    ms = c4_sizes(count)
    jobs = [(s, ms[s]) for s in (range(count) if which is None else which)]
    with mp.get_context("spawn").Pool(min(os.cpu_count() or 1, 32)) as pool:
        return pool.map(_c4_system, jobs, chunksize=8)


def shard_by_work(work, world):
    """Independent systems over `world` GPUs with no exchange: largest estimated work first, each to
    the least-loaded rank (ties: lowest index, lowest rank).  Returns each rank's sorted indices."""
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for s in sorted(range(len(work)), key=lambda i: (-float(work[i]), i)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(s)
        load[r] += float(work[s])
    return [sorted(p) for p in parts]


def run_c4(args):
    """2,000 independent Delaunay systems factored as one batch (level launches over the merged task lists),
    FP32 factor + FP64 refinement to max(1e-10, 2 x the residual the reference's FP64 code attains on the
    batch), 1 RHS each.  When the refinement breaks down on a system
    whose conditioning is beyond FP32, the handle falls back to an FP64 factor (reported in the line)."""
    count = args.batch or C4_COUNT
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    # several GPUs: the systems shard by estimated factor work (~m^1.5 for a 2D mesh under nested
    # dissection), no collective on the data path
    mine = shard_by_work(c4_sizes(count).astype(np.float64) ** 1.5, world)[rank] if world > 1 else None
    systems = c4_systems(count, mine)                  # process pool before any GPU call
    import torch
    from tensors_b200 import build as tb_build
    from tensors_b200.cholesky import BatchedCholesky

    tb_build.build()
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        torch.cuda.set_device(dev)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)
    t0 = time.perf_counter()
    b = BatchedCholesky([(o, i, p) for o, i, v, p in systems])
    b.handle.SetSchedule(args.schedule or "levels")
    b.handle.SymbolicFactorization()
    t_setup = time.perf_counter() - t0
    vals = torch.tensor(np.concatenate([v for o, i, v, p in systems]), device=dev)
    n = int(b.row_offsets[-1])
    B = torch.tensor(np.random.default_rng(C4_SEED + 1).standard_normal(n), device=dev)
    X = torch.empty_like(B)
    stream = torch.cuda.Stream(dev)
    b.handle.SetStream(stream)
    torch.cuda.set_stream(stream)
    # Untimed: the residual a plain FP64 factor + solve attains on this batch, on the GPU and with the
    # reference's own CPU code.  On the worst meshes (kappa ~1e14) the FP64 floor u |A| |x| / |b| lies
    # far above 1e-10, so the refinement target is max(1e-10, 2 x the reference's attainable residual).
    b.handle.SetPrecision("fp64")
    assert b.NumericFactorization(vals, 0.0) == 0
    b.Solve(B, X)
    attainable = float(torch.linalg.norm(b.handle.Residual(B, X)) / torch.linalg.norm(B))
    ref = None
    if not args.no_cpu_baseline and world == 1:
        ref = c4_reference(systems, B.cpu().numpy(), np.asarray(b.row_offsets), X.cpu().numpy())
    target = max(TARGET_RELRES, 2.0 * (ref["relres"] if ref else attainable))
    b.handle.SetPrecision("mixed")
    b.handle.SetRefinement(target, 60)

    def step(mid):
        assert b.NumericFactorization(vals, 0.0) == 0
        if mid is not None:
            mid.record(stream)
        b.Solve(B, X)

    with ClockSampler(local) as clocks:
        t, tf = _time_steps(torch, stream, step, args.steps, args.warmup,
                            barrier=dist.barrier if dist is not None else None)
    stream.synchronize()
    it, rr = b.handle.RefinementInfo()
    R = b.handle.Residual(B, X)
    stream.synchronize()
    relres = float(torch.linalg.norm(R) / torch.linalg.norm(B))
    F, nnz_u = b.handle.FlopCount()
    flops = F + 4.0 * nnz_u
    n_systems = len(systems)
    if dist is not None:
        # the job: every rank's work over the slowest rank's time
        t, tf = max_over_ranks(dist, t, dev), max_over_ranks(dist, tf, dev)
        relres, target = max_over_ranks(dist, relres, dev), max_over_ranks(dist, target, dev)
        tot = torch.tensor([flops, F, float(n_systems), float(n)], dtype=torch.float64, device=dev)
        dist.all_reduce(tot)
        flops, F, n_systems, n = float(tot[0]), float(tot[1]), int(tot[2]), int(tot[3])
        dist.barrier()
        dist.destroy_process_group()
        if rank != 0:
            return 0
    line = {
        "metric": f"batched factor+solve GFLOP/s, {n_systems} Delaunay systems, FP32 factor + FP64 refinement "
                  f"to max({TARGET_RELRES:g}, 2 x the reference's FP64 residual)",
        "value": flops / (t * 1e-3) / 1e9, "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic (seeded)",
        "config": {"workload": f"{n_systems} 2D Delaunay meshes, m ~ U[{C4_MIN}, {C4_MAX}] points, cotangent "
                               "Laplacian + 1e-3 lumped mass, nested dissection each, 1 RHS each",
                   "parallelism": f"{world} GPU(s), systems sharded by estimated factor work, no collective",
                   "rows": n, "factor_gflop": F / 1e9, "factor_ms": tf, "solve_ms": t - tf,
                   "systems_per_s": n_systems / (t * 1e-3), "refinement": [it, rr], "relres": relres,
                   "target": target, "target_from": "reference CPU residual" if ref else "GPU FP64 residual",
                   "fp64_direct_relres": attainable,
                   "reference_relres": ref["relres"] if ref else None,
                   "worst_gpu_over_reference_relres": ref["worst_ratio"] if ref else None,
                   "perturbed_pivots": b.handle.PerturbedPivots(),
                   "precision_in_use": list(b.handle.PrecisionInUse()),
                   "schedule": args.schedule or "levels", "setup_s": t_setup,
                   "plan": b.handle.PlanStats(), "clocks": clocks.summary()},
        "cpu_baseline": None if ref is None else {
            "value": flops / ref["seconds"] / 1e9, "unit": "GFLOP/s", "cores": ref["cores"], "kind": "reference",
            "sample": "the reference's own code on every system of the batch, one factor + solve each "
                      "(all host threads per system)", "seconds": ref["seconds"]},
    }
    print(json.dumps(line))
    return 0


def c4_reference(systems, B, offsets, X_gpu):
    """The reference's own CPU factor + solve of every system of the batch: the stacked relative residual it
    attains, the worst ratio of the GPU FP64 solution's per-system residual to the reference's, and its time."""
    import scipy.sparse as sp

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    if not oracle.ref_available():
        return None
    threads = os.cpu_count() or 1
    r2 = b2 = 0.0
    secs = 0.0
    worst = 0.0
    for s, (outer, inner, values, perm) in enumerate(systems):
        n = len(outer) - 1
        o0, o1 = int(offsets[s]), int(offsets[s + 1])
        bs = np.ascontiguousarray(B[o0:o1])
        ref = oracle.RefCholesky(n, outer, inner, perm, "maximal", threads=threads, blas_threads=1)
        ref.symbolic()
        t0 = time.perf_counter()
        ref.factor(values, 0.0)
        xs = ref.solve(bs, parallel=False)
        secs += time.perf_counter() - t0
        A = sp.csr_matrix((values, inner, outer), shape=(n, n))
        rr = float(np.linalg.norm(bs - A @ xs) ** 2)
        rg = float(np.linalg.norm(bs - A @ X_gpu[o0:o1]) ** 2)
        r2 += rr
        b2 += float(np.linalg.norm(bs) ** 2)
        if rr > 0.0:
            worst = max(worst, np.sqrt(rg / rr))
        del ref
    return {"relres": float(np.sqrt(r2 / b2)), "worst_ratio": float(worst), "seconds": secs, "cores": threads}


# Arrival rate below the measured service capacity (about 43 requests/s with 4
# slots: a 64^3 request with 64 RHS runs ~0.1 s), so latencies measure the
# served stream rather than an unbounded queue.  The full 10,000-request
# stream takes about 5.5 minutes at this rate (--requests 10000); the default
# bench run serves the first 2,000 requests of the same stream.
C5_REQUESTS, C5_RATE, C5_SEED, C5_CAP, C5_SLOTS, C5_POOL = 2000, 30.0, 0x5EED0005, 150 << 30, 4, 32


def _c5_matrix(args):
    j, kind, g = args
    from tensors_b200 import matrices, ordering

    # 2D: a quality mesh of about g^2 points (jittered grid, Delaunay, cotangent Laplacian + the
    # lumped mass scaled to a mean diagonal shift of 1e-2, the 2D generator's shift; an absolute
    # 1e-3 x mass of ~1/g^2 puts kappa near 1e8 on the largest meshes, where even FP64 stalls
    # near 4e-9 against the 1e-10 target); 3D: the 7-point grid Laplacian of a g^3 grid with
    # lognormal conductivities
    A = (matrices.mesh_laplacian(int(g) * int(g), C5_SEED + j, 1e-2, relative=True) if kind == "2d"
         else matrices.grid_laplacian_3d(int(g), C5_SEED + j, 1e-2))
    return kind, int(g), A.outer, A.inner, A.values, ordering.nested_dissection(A)


def c5_reference_time(mats, which, repeat, nrhs, reqs):
    """The reference's own CPU code on the served requests: each pool matrix factored once and solved
    with 1 and with 64 right-hand sides on all host threads (symbolic analysis untimed, as the server's
    warm-up); a request costs its matrix's factor time (unless it is a repeat solve) plus its solve time
    interpolated linearly in its RHS count.  Returns the summed busy time and the throughput it allows."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle

    if not oracle.ref_available():
        return None
    threads = os.cpu_count() or 1
    per = {}
    for j, (kind, g, outer, inner, values, perm) in mats.items():
        n = len(outer) - 1
        ref = oracle.RefCholesky(n, outer, inner, perm, "maximal", threads=threads, blas_threads=1)
        ref.symbolic()
        t0 = time.perf_counter()
        ref.factor(values, 0.0)
        tf = time.perf_counter() - t0
        ts = []
        for k in (1, 64):
            B = np.random.default_rng(j).standard_normal((n, k))
            t0 = time.perf_counter()
            ref.solve(B, parallel=False)
            ts.append(time.perf_counter() - t0)
        per[j] = (tf, ts[0], ts[1])
        del ref
    total = 0.0
    for r in reqs:
        tf, s1, s64 = per[int(which[r])]
        k = int(nrhs[r])
        total += (0.0 if repeat[r] else tf) + s1 + (s64 - s1) * (k - 1) / 63.0
    return {"value": len(reqs) / total, "unit": "requests/s", "cores": threads, "kind": "reference",
            "sample": "the reference's own code: every pool matrix factored once and solved with 1 and 64 RHS, "
                      "summed over the stream's requests (factor unless a repeat solve, solve interpolated in k)",
            "busy_s": total, "factor_s_per_matrix": {str(j): v[0] for j, v in per.items()}}


def run_setup(args):
    """Host set-up of the C2 and C3 systems (no GPU): both nested-dissection orderings, the
    symbolic analysis by phase (the phase ranges' host times), the device plan and the plan
    check, each the median of --steps runs.  One JSON line."""
    import statistics

    from tensors_b200 import build as tb_build
    from tensors_b200 import matrices, ordering, trace
    from tensors_b200.cholesky import CholeskyDecomposition

    tb_build.build()
    P = "Sparse::CholeskyDecomposition::"
    phases = [("init", P + "Init"), ("elimination_tree", P + "EliminationTree"), ("postordering", P + "PostOrdering"),
              ("supernodes", P + "FindMaximalSupernodes"), ("supernode_starts", "tensors_b200::SupernodeStarts"),
              ("assembly_tree", P + "CreateAssemblyTree"),
              ("analysis", P + "SymbolicFactorization"), ("plan", "tensors_b200::DevicePlan")]
    systems = {"c2": (f"3D 7-point Laplacian {GRID}^3", lambda: matrices.grid_laplacian_3d(GRID, SEED, SHIFT)),
               "c3": (f"3-dof 27-point vector Laplacian {C3_GRID}^3",
                      lambda: matrices.vector_laplacian_3d(C3_GRID, C3_SEED, C3_SHIFT))}
    steps = max(1, args.steps)
    out = {}
    for key, (name, make) in systems.items():
        A = make()
        rec = {"n": A.n, "nnz": int(A.outer[-1])}
        for oname, fn in (("geometric", ordering.nested_dissection), ("graph", ordering.graph_nested_dissection)):
            ts = []
            for _ in range(steps):
                t0 = time.perf_counter()
                perm = fn(A)
                ts.append(1e3 * (time.perf_counter() - t0))
            rec[f"ordering_{oname}_ms"] = statistics.median(ts)
        perm = ordering.graph_nested_dissection(A) if key == "c2" else ordering.nested_dissection(A)
        got = {k: [] for k, _ in phases}
        got["plan_check"] = []
        for _ in range(steps):
            trace.record(True)
            try:
                c = CholeskyDecomposition(A.outer, A.inner, perm)
                c.SymbolicFactorization()
                times = dict(trace.times())
            finally:
                trace.record(False)
            for k, tag in phases:
                got[k].append(times.get(tag, float("nan")))
            t0 = time.perf_counter()
            c.CheckPlan()
            got["plan_check"].append(1e3 * (time.perf_counter() - t0))
        stats = c.PlanStats()
        # the SymbolicFactorization range holds the plan build: analysis = the range less the plan;
        # a phase that did not run (PostOrdering of an ordering already postordered) is null
        got["analysis"] = [a - p for a, p in zip(got["analysis"], got["plan"])]
        rec.update({f"{k}_ms": (None if any(x != x for x in v) else statistics.median(v)) for k, v in got.items()})
        rec.update({"fronts": stats["fronts"], "gemm_tasks": stats["gemm_tasks"], "supernodes": stats["supernodes"]})
        out[key] = rec
    line = {"metric": "host set-up time (ordering, symbolic analysis, device plan, plan check)", "unit": "ms",
            "value": out["c2"]["analysis_ms"] + out["c2"]["plan_ms"], "higher_is_better": False,
            "steps": steps, "cores": os.cpu_count(), "data": "synthetic (seeded)",
            "config": {"workload": "C2 and C3 systems, median of steps", "systems": out}}
    print(json.dumps(line))
    return 0


def run_c5(args):
    """Serving: a Poisson stream of factor / solve requests over a pool of 2D mesh Laplacians
    (quality meshes, n 1k-50k) and 3D 7-point grids (32^3-64^3), 1-64 RHS each, 30% solves on
    resident factors, 150 GB HBM cap, FP32 factor + FP64 refinement to 1e-10; reports p50 / p99
    latency and throughput, and the reference's CPU time for the same requests (each matrix's
    factor and solve timed once on the host, summed over the stream's requests)."""
    import multiprocessing as mp

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    rng = np.random.default_rng(C5_SEED)
    half = C5_POOL // 2
    specs = [(j, "2d", int(rng.integers(32, 224 + 1))) for j in range(half)]
    specs += [(half + j, "3d", int(rng.integers(32, 64 + 1))) for j in range(C5_POOL - half)]
    # several GPUs: the matrices (and with them their requests) shard by estimated factor work,
    # g^3 for a 2D g x g grid and g^6 for a 3D g^3 grid under nested dissection; no collective
    # on the data path, latencies gathered at the end
    mine = (shard_by_work([float(g) ** (3 if kind == "2d" else 6) for _, kind, g in specs], world)[rank]
            if world > 1 else list(range(len(specs))))
    with mp.get_context("spawn").Pool(min(os.cpu_count() or 1, len(mine), 16)) as pool:     # before any GPU call
        mats = dict(zip(mine, pool.map(_c5_matrix, [specs[j] for j in mine])))
    from tensors_b200 import build as tb_build
    from tensors_b200.serving import Server

    tb_build.build()
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    n_req = args.requests or C5_REQUESTS
    srv = Server(hbm_cap_bytes=C5_CAP, slots=C5_SLOTS, precision="mixed", device=local)
    ids = {j: srv.add_matrix(m[2], m[3], m[5]) for j, m in mats.items()}
    blocks = {j: np.random.default_rng(C5_SEED + 100 + j).standard_normal((len(m[2]) - 1, 64)) for j, m in mats.items()}
    # warm-up: symbolic analysis, device plan and first factor of every matrix (the reference's
    # SymbolicFactorization precedes NumericFactorization in the same way), then one solve per
    # right-hand-side width class (the solves run on 8, 16, 32 or 64 columns: each class's
    # graph is captured and its buffers sized once); its time is reported as cold_start_s
    t_cold = time.perf_counter()
    for t in [srv.submit(ids[j], values=mats[j][4], B=blocks[j][:, :1].copy(), tol=TARGET_RELRES) for j in mine]:
        srv.wait(t)
    for width in (16, 32, 64):
        for t in [srv.submit(ids[j], B=np.ascontiguousarray(blocks[j][:, :width]), tol=TARGET_RELRES) for j in mine]:
            srv.wait(t)
    cold_start = time.perf_counter() - t_cold
    arrivals = np.cumsum(rng.exponential(1.0 / C5_RATE, size=n_req))
    which = rng.integers(0, len(specs), size=n_req)
    repeat = rng.random(n_req) < 0.3
    nrhs = rng.integers(1, 65, size=n_req)
    scales = 1.0 + 0.1 * rng.random(n_req)
    owned = set(mine)
    reqs = [r for r in range(n_req) if int(which[r]) in owned]     # this rank's share of the stream
    tickets = {r: None for r in reqs}
    import threading as th

    if dist is not None:
        dist.barrier()
    start = time.perf_counter()

    def submitter():
        for r in reqs:
            delay = start + arrivals[r] - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            j = int(which[r])
            B = np.ascontiguousarray(blocks[j][:, : int(nrhs[r])])
            vals = None if repeat[r] else mats[j][4] * scales[r]
            tickets[r] = srv.submit(ids[j], values=vals, B=B, tol=TARGET_RELRES)

    sub = th.Thread(target=submitter)
    sub.start()
    lat, runs, iters, worst, fails = [], [], [], 0.0, 0
    for r in reqs:
        while tickets[r] is None:
            time.sleep(0.0005)
        X, info = srv.wait(tickets[r])
        if info["status"] != 0:
            fails += 1
        lat.append(info["latency_ms"])
        runs.append(info["run_ms"])
        iters.append(info["iterations"])
        worst = max(worst, info["relres"])
        tickets[r] = True
    sub.join()
    wall = time.perf_counter() - start
    st = srv.stats()
    srv.close()
    if dist is not None:
        # the job's latency distribution: every rank's requests, over the slowest rank's wall time
        parts = [None] * world
        dist.all_gather_object(parts, (lat, runs, iters, worst, fails, wall, cold_start))
        lat = [x for p in parts for x in p[0]]
        runs = [x for p in parts for x in p[1]]
        iters = [x for p in parts for x in p[2]]
        worst = max(p[3] for p in parts)
        fails = sum(p[4] for p in parts)
        wall = max(p[5] for p in parts)
        cold_start = max(p[6] for p in parts)
        dist.barrier()
        dist.destroy_process_group()
        if rank != 0:
            return 0
    lat = np.array(lat)
    ref = None
    if not args.no_cpu_baseline and world == 1:
        ref = c5_reference_time(mats, which, repeat, nrhs, reqs)
    line = {
        "metric": "serving latency p50/p99 (ms) and throughput, Poisson stream of factor/solve requests, "
                  "FP32 factor + FP64 refinement to 1e-10",
        "value": float(np.percentile(lat, 99)), "unit": "ms (p99 latency)", "n_gpus": world, "steps": n_req,
        "warmup": 4 * len(specs), "ms_per_step": float(np.mean(runs)), "higher_is_better": False, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded)",
        "config": {"workload": f"{n_req} requests, Poisson arrivals at {C5_RATE:g}/s over {len(specs)} matrices "
                               "(2D quality-mesh cotangent Laplacians n 1k-50k + mass-weighted shift of mean 1e-2, 3D 7-point "
                               "grids 32^3-64^3), 1-64 RHS, 30% "
                               "solves on resident factors, 150 GB HBM cap, 4 slots",
                   "p50_ms": float(np.percentile(lat, 50)), "p90_ms": float(np.percentile(lat, 90)),
                   "p99_ms": float(np.percentile(lat, 99)), "mean_run_ms": float(np.mean(runs)),
                   "parallelism": f"{world} GPU(s), matrices and their requests sharded by estimated factor work",
                   "throughput_req_per_s": n_req / wall, "wall_s": wall, "failures": fails,
                   "cold_start_s": cold_start,
                   "warmup_note": "untimed: per matrix the symbolic analysis, plan and first factor, then one solve "
                                  "per right-hand-side width class (16, 32, 64 columns)",
                   "worst_relres": worst, "mean_refinement_steps": float(np.mean(iters)), "server": st},
        "cpu_baseline": ref,
    }
    print(json.dumps(line))
    return 0


def max_over_ranks(dist, value, device):
    """The largest of the ranks' values, on every rank (one all-reduce)."""
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(flops_per_replica, t_ms, world):
    """Whole-job GFLOP/s of `world` independent replicas, each doing
    flops_per_replica per step, timed by the slowest rank's t_ms."""
    return flops_per_replica / (t_ms * 1e-3) / 1e9 * world


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--grid", type=int, default=GRID, help="grid edge (profiling runs on smaller cases)")
    ap.add_argument("--workload", default="c2", choices=["c2", "c3", "c4", "c5", "setup"],
                    help="c2 (default): the headline FP64 64^3 Laplacian; c3: mixed vs FP64 vector Laplacian; "
                         "c4: batched Delaunay systems; c5: serving stream; setup: host set-up phases (no GPU)")
    ap.add_argument("--batch", type=int, default=0, help="c4: number of systems (default 2000)")
    ap.add_argument("--requests", type=int, default=0, help="c5: number of requests (default 2000 of the 10000)")
    ap.add_argument("--schedule", default=None, help="c4: factorization schedule of the batch")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="--ncu runs: factor precision (mixed: FP32 factor with tensor-core GEMM tiles)")
    ap.add_argument("--ncu", action="store_true",
                    help="profiling run for ncu: warmup + steps factor+solve as direct launches, no timing, "
                         "no baselines")
    ap.add_argument("--ordering", default="graph", choices=["geometric", "graph"],
                    help="c2: nested dissection from the pattern alone (default: fewer factor flops on this grid) "
                         "or from the node coordinates (GFLOP/s is computed from each ordering's own flops)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default plan options instead of the autotuner's choice (untimed set-up)")
    ap.add_argument("--no-mixed", action="store_true",
                    help="c2: skip the mixed-precision vs FP64 comparison on the 48^3 vector Laplacian")
    ap.add_argument("--c3-steps", type=int, default=5, help="timed steps of each precision in that comparison")
    args = ap.parse_args()
    global ORDERING
    ORDERING = args.ordering
    if args.impl == "reference":
        return run_reference(args)
    if args.ncu:
        return run_for_profiler(args)
    if args.workload == "c3":
        return run_c3(args)
    if args.workload == "c4":
        return run_c4(args)
    if args.workload == "c5":
        return run_c5(args)
    if args.workload == "setup":
        return run_setup(args)

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)

    from tensors_b200 import build as tb_build
    from tensors_b200._lib import lib
    from tensors_b200.cholesky import CholeskyDecomposition

    tb_build.build()
    lib().tb_set_device(local)

    A, perm, B_host = build_problem()
    t0 = time.perf_counter()
    chol = CholeskyDecomposition(A.outer, A.inner, perm)
    chol.SymbolicFactorization()
    t_symbolic = time.perf_counter() - t0
    F, nnz_u = chol.FlopCount()
    flops = F + 4.0 * NRHS * nnz_u

    vals = torch.tensor(A.values, device=dev)
    B = torch.tensor(B_host, device=dev)
    X = torch.empty_like(B)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    # one dedicated stream for the library's kernels, the L2 flush and the events
    stream = torch.cuda.Stream(dev)
    chol.SetStream(stream)
    torch.cuda.set_stream(stream)

    def step():
        st = chol.NumericFactorization(vals, 0.0)
        chol.Solve(B, X)
        return st

    # untimed set-up: the library's plan autotuner picks the trailing-update deferral and the front
    # relaxation for this matrix by timing its own factorizations (the work counted in the metric is
    # the reference's supernodes' flops, whatever the choice)
    tuned = None
    if not args.no_autotune:
        assert chol.NumericFactorization(vals, 0.0) == 0
        tuned = chol.AutotunePlan()["choice"]
    for _ in range(args.warmup):
        assert step() == 0
    torch.cuda.synchronize(dev)

    times, factor_times = [], []
    with ClockSampler(local) as clocks:
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        for _ in range(args.steps):
            flush.fill_(1.0)
            s, m, e = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            s.record(stream)
            chol.NumericFactorization(vals, 0.0)
            m.record(stream)
            chol.Solve(B, X)
            e.record(stream)
            e.synchronize()
            times.append(s.elapsed_time(e))
            factor_times.append(s.elapsed_time(m))
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
    t_ms = statistics.mean(times)
    if world > 1:
        t_ms = max_over_ranks(dist, t_ms, dev)

    # correctness of the timed result
    R = chol.Residual(B, X)
    torch.cuda.synchronize(dev)
    relres = float(torch.linalg.norm(R) / torch.linalg.norm(B))
    fl, sl = chol.LaunchCounts()

    # end to end through the host-buffer C-ABI calls (copies inside the timing)
    Xh = np.zeros_like(B_host)
    e2e = []
    for i in range(max(2, min(args.steps, 3)) + 1):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        chol.NumericFactorization(A.values, 0.0)
        chol.Solve(B_host, Xh)
        dt = time.perf_counter() - t0
        if i > 0:
            e2e.append(dt)
    e2e_s = statistics.mean(e2e)

    # per-kernel timing of the GEMM tiles (direct launches with events)
    chol.SetProfiling(True)
    prof = None
    for _ in range(2):
        chol.NumericFactorization(vals, 0.0)
        prof = chol.KernelProfile()
    chol.SetProfiling(False)
    dgemm_peak = measure_dgemm_tflops(torch, dev)
    plan_stats = chol.PlanStats()
    F_geo = None
    if ORDERING != "geometric" and rank == 0:
        cg = CholeskyDecomposition(A.outer, A.inner, c2_permutation(A, "geometric"))
        F_geo = cg.FlopCount()[0]
        del cg

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return 0

    g = prof["gemm"]
    achieved = g["flops"] / (g["ms"] * 1e-3) / 1e12 if g["ms"] > 0 else None
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "gemm_tn_traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get("bytes_per_launch")
        except Exception:
            traffic = None

    cpu = None
    if not args.no_cpu_baseline and world == 1:
        # the reference's own code on the same system (same ordering, values and RHS), all host threads
        threads = os.cpu_count() or 1
        r = reference_run(A, perm, B_host, threads, steps=1, warmup=0)
        if r is not None:
            Xg = X.cpu().numpy()
            cpu = {"value": r["flops"] / r["seconds"][0] / 1e9, "unit": "GFLOP/s", "cores": threads,
                   "kind": "reference",
                   "sample": f"the reference's own code, one factor+solve of the benchmark system "
                             f"({threads} tree threads, 1 BLAS thread each)",
                   "seconds": r["seconds"][0], "relres": r["relres"],
                   "forward_diff_vs_gpu": float(np.linalg.norm(Xg - r["X"]) / np.linalg.norm(r["X"]))}
            del r
            if ORDERING != "geometric":
                # the same reference run under the geometric dissection (twice the flops on this grid)
                Ag, pg, Bg = build_problem(args.grid, "geometric")
                rg = reference_run(Ag, pg, Bg, threads, steps=1, warmup=0)
                cpu["geometric_ordering"] = {"value": rg["flops"] / rg["seconds"][0] / 1e9, "unit": "GFLOP/s",
                                             "seconds": rg["seconds"][0], "factor_gflop": rg["factor_flops"] / 1e9,
                                             "relres": rg["relres"]}
                del rg

    mixed = None
    if not args.no_mixed and world == 1:
        del chol
        torch.cuda.empty_cache()
        mixed = c3_compare(torch, dev, args.c3_steps, args.warmup, not args.no_autotune)

    value = replica_throughput(flops, t_ms, world)
    line = {
        "metric": METRIC,
        "value": value, "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded)",
        "config": config_dict({
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "plan_options": {"defer_steps": tuned[0], "relax": tuned[1], "tc_width": tuned[2],
                             "chosen_by": "tb_chol_autotune_plan (untimed set-up)"} if tuned else "defaults",
            "relres": relres, "symbolic_s": t_symbolic,
            "factor_ms": statistics.mean(factor_times), "solve_ms": t_ms - statistics.mean(factor_times),
            "factor_gflop": F / 1e9, "solve_gflop": 4.0 * NRHS * nnz_u / 1e9,
            "plan": plan_stats,
            "kernel_ms": {k: round(v["ms"], 3) for k, v in prof.items()},
            "flops_geometric_ordering_gflop": F_geo / 1e9 if F_geo else None,
            "mixed_vs_fp64": mixed,
        }),
        "e2e": {"value": flops / e2e_s / 1e9 * world, "unit": "GFLOP/s",
                "h2d_bytes_per_step": int(A.values.nbytes + B_host.nbytes),
                "d2h_bytes_per_step": int(B_host.nbytes), "ms_per_step": e2e_s * 1e3},
        "roofline": {"bound": "tensor", "kernel": "gemm_tn_kernel (FP64 DMMA tiles)",
                     "achieved": achieved, "peak": dgemm_peak, "unit": "TFLOP/s",
                     "frac": (achieved / dgemm_peak) if achieved else None, "traffic": traffic,
                     "peak_source": "measured live: cuBLAS FP64 GEMM 8192^3 (MEASURED_PEAKS.json has no FP64 figure)"},
        "cpu_baseline": cpu,
        "clocks": clocks.summary(),
        "gpu_launches": int((fl + sl) * args.steps),
    }
    print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
