"""The multi-rank host logic of bench.py on the CPU: two gloo ranks (world_size 2, 127.0.0.1).

bench.py runs one process per GPU. The single-cavity workload runs one replica per rank. The
batched workload shards the cavities with a size-balanced partition and no data-path collective.
torch.distributed serves only for the barrier and the max over ranks. Here two CPU ranks check:
* the shards of the 256-cavity manifest are disjoint, cover it, and balance the N^3 cost;
* allmax returns the slowest rank's time on every rank;
* the barrier completes.
"""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

REPO = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(REPO))
    import datetime
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        manifest = bench.batch_manifest(256, 20261203)
        mine = bench.batch_shard(manifest, world, rank)
        shards = [None] * world
        dist.all_gather_object(shards, mine)
        slowest = bench.allmax(float(rank + 1) * 1.5, world)
        bench.barrier(world)
        out.put((rank, shards, slowest))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sys.path.insert(0, str(REPO))
    import bench
    manifest = bench.batch_manifest(256, 20261203)
    for rank, shards, slowest in res:
        assert slowest == 3.0  # rank 1's 2 x 1.5
        a, b = set(shards[0]), set(shards[1])
        assert not (a & b) and (a | b) == set(range(256))
        cost = [sum(manifest[i][0] ** 3 for i in sh) for sh in shards]
        assert max(cost) / min(cost) < 1.01
