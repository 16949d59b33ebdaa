"""The multi-GPU bench path without GPUs: N independent replicas, timed by the
slowest rank (max over ranks), whole-job throughput = N x one replica's work
over that time; the reference arm runs on rank 0 only.  Two gloo ranks on
CPU stand in for two GPUs.  The batch workload's partition of systems over
ranks is checked directly."""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = 10.0 + 5.0 * rank                    # rank 1 is the slow one
        t = bench.max_over_ranks(dist, local_ms, "cpu")
        dist.barrier()
        out.put((rank, t, bench.replica_throughput(2.0e9, t, world)))
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_slowest_rank_and_sum_the_work():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in procs)
    assert [r[1] for r in res] == [15.0, 15.0]
    # 2 replicas x 2 GFLOP in 15 ms
    assert all(abs(r[2] - 2 * 2.0 / 0.015) < 1e-6 for r in res)


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == ""


def test_replica_throughput_is_linear_in_ranks():
    assert bench.replica_throughput(1e9, 1000.0, 1) == pytest.approx(1.0)
    assert bench.replica_throughput(1e9, 1000.0, 8) == pytest.approx(8.0)
    json.dumps({"v": bench.replica_throughput(3e9, 7.0, 4)})


def test_batch_shards_cover_every_system_once_and_balance_the_work():
    rng = np.random.default_rng(0)
    work = rng.integers(1, 1000, 137).astype(float)
    for world in (1, 2, 3, 8):
        parts = bench.shard_by_work(work, world)
        assert len(parts) == world
        assert sorted(i for p in parts for i in p) == list(range(len(work)))
        assert all(p == sorted(p) for p in parts)
        loads = [work[p].sum() for p in parts]
        assert max(loads) - min(loads) <= work.max()           # greedy largest-first bound
        assert parts == bench.shard_by_work(work, world)        # deterministic
    # the C4 batch over 2-8 GPUs: within 1% of an even split
    w = bench.c4_sizes(2000).astype(float) ** 1.5
    for world in (2, 4, 8):
        loads = [w[p].sum() for p in bench.shard_by_work(w, world)]
        assert max(loads) / (w.sum() / world) < 1.01


def test_a_rank_generates_exactly_its_share_of_the_batch():
    # systems are seeded by their index in the whole batch, so a rank's subset equals the full batch's rows
    full = bench.c4_systems(4)
    part = bench.c4_systems(4, [1, 3])
    for got, want in zip(part, [full[1], full[3]]):
        for a, b in zip(got, want):
            assert np.array_equal(a, b)
