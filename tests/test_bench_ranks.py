"""bench.py's multi-rank host logic on CPU (gloo, world size 2): the
max-over-ranks timing reduction and the broadcast of rank 0's tuned choice
that every replica runs."""
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


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mx = bench.max_over_ranks([1.0 + rank, 5.0 - rank], world, "cpu")
        r0 = bench.from_rank0([8.0 if rank == 0 else 2.0, 148.0 * (rank + 1)], world, "cpu")
        q.put((rank, mx, r0))
    finally:
        dist.destroy_process_group()


def test_rank_reductions_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, mx, r0 in got:
        assert mx == [2.0, 5.0]
        assert r0 == [8.0, 148.0]


def test_single_rank_identity():
    assert bench.max_over_ranks([3, 4.5], 1, "cpu") == [3.0, 4.5]
    assert bench.from_rank0([16, 0], 1, "cpu") == [16.0, 0.0]
