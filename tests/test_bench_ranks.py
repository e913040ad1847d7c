"""bench.py's multi-rank path on CPU: two gloo ranks (the replica layout
torchrun gives bench.py --gpus 2) agree on the slowest rank's time and on
the whole-job throughput, with no data-path collective (replicas only)."""

from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = [120.0, 180.5][rank]  # each replica's own device time
        ms = bench.max_over_ranks(local_ms, dist)
        value = bench.replica_throughput(ms, world, cells=1000, nsub=10, steps=4)
        dist.barrier()
        q.put((rank, ms, value))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, ms, value in got:
        assert ms == 180.5
        assert value == pytest.approx(2 * 1000 * 10 * 4 / 0.1805)


def test_single_rank_is_its_own_time():
    assert bench.max_over_ranks(12.5) == 12.5
    assert bench.replica_throughput(1000.0, 1, 10, 10, 1) == 100.0
