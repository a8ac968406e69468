"""The multi-rank host logic of bench.py on CPU: two `gloo` ranks (127.0.0.1).

Each rank runs its own seeded instance (weak scaling, no data-path
collective); the job time is the max over ranks and the whole-job rate counts
every rank's units.  Also: the reference arm's non-zero ranks exit without
work."""
import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local = 1.5 + rank            # rank 1 is the slow one
        tmax = bench.max_over_ranks(local, world, dist, "cpu")
        rate = bench.job_rate(100.0, world, tmax)
        x, _, _, _ = bench.make_inputs(64, bench.rank_seed(7, rank))
        q.put((rank, tmax, rate, float(x.sum())))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_time_is_max_and_rate_counts_all_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, t0, v0, s0), (r1, t1, v1, s1) = res
    assert t0 == t1 == 2.5                      # slowest rank
    assert v0 == v1 == pytest.approx(2 * 100.0 / 2.5)
    assert s0 != s1                             # each rank sweeps its own instance


def test_single_rank_needs_no_collective():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.0, 1) == 3.0
    assert bench.job_rate(10.0, 1, 2.0) == 5.0


def test_reference_arm_nonzero_rank_exits_without_work(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")

    class A:
        n, seed, steps, warmup = 1024, 1, 1, 1
    assert bench.run_reference(A()) == 0
