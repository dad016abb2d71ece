"""The multi-rank plumbing of bench.py (replicas, one process per GPU) with two
`gloo` ranks on the CPU: process-group set-up, the timing barrier and the
max-over-ranks reduction that makes the slowest replica set the job's time,
and the whole-job throughput."""
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch
    import bench
    dist = bench.init_ranks(world, rank, backend="gloo", timeout_s=30)
    try:
        dist.barrier()
        # rank r "took" 10 + r ms for 100 steps of a 1000-cell case
        t_ms = bench.max_over_ranks(10.0 + rank, dist, torch.device("cpu"))
        rate = bench.job_throughput(world, 1000 * 100, t_ms / 1000.0)
        q.put((rank, t_ms, rate))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_replica():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, t_ms, rate in got:
        assert t_ms == 11.0                         # max over ranks
        assert rate == pytest.approx(2 * 1000 * 100 / 0.011)


def test_single_rank_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.init_ranks(1, 0) is None
    assert bench.max_over_ranks(3.5, None, None) == 3.5
    assert bench.job_throughput(1, 500, 0.5) == 1000.0
