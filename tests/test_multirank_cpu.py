"""The N>1 path of bench.py (replicas, one process per GPU) on the CPU with
gloo, world_size 2: ranks get disjoint right-hand sides, the timing taken is
the max over ranks, and the barrier joins both ranks."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    import datetime

    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    seeds = {bench.rank_rhs_seed(rank, i, c) for i in range(4) for c in range(64)}
    t = bench.max_over_ranks(1.5 + rank, world)
    bench.barrier(world)
    q.put((rank, t, sorted(seeds)[:3], len(seeds)))
    dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert out[0][1] == out[1][1] == 2.5  # slowest rank wins
    seeds0 = {bench_seed for bench_seed in out[0][2]}
    seeds1 = {bench_seed for bench_seed in out[1][2]}
    assert not (seeds0 & seeds1)
    assert out[0][3] == out[1][3] == 256
