"""The multi-rank arithmetic of bench.py on two gloo ranks (CPU): every rank gets the slowest rank's
time, and the whole-job rate counts every replica's cells against that time."""

import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 10.0 * (rank + 1)  # rank 1 is the slow one
        slowest = bench.max_over_ranks(ms, dist)
        dist.barrier()
        out.put((rank, slowest, bench.whole_job_rate(1000, 5, world, slowest / 1000.0)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [20.0, 20.0]
    assert res[0][2] == pytest.approx(1000 * 5 * 2 / 0.02)


def test_single_rank_needs_no_group():
    assert bench.max_over_ranks(3.5, None) == 3.5
