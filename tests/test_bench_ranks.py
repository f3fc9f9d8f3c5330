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


def test_reference_arm_json_contract():
    """`bench.py --impl reference` (the reference's own cpu_solver on the host
    cores) prints one JSON line with the contract's keys, on a small grid."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    import oracle
    if not oracle.ref_available():
        pytest.skip("reference library not built")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--grid", "16", "--steps", "1",
                        "--warmup", "3"], capture_output=True, text=True, cwd=root, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    d = json.loads(r.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference" and d["unit"] == "solves/s" and d["value"] > 0
    assert d["steps"] == 1 and d["warmup"] == 3 and d["n_gpus"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert "fit in L2" in d["config"]["l2"]
