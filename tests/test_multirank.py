"""bench.py's multi-GPU logic on CPU: replicas reduce their device times with
a MAX over ranks (gloo, world size 2, 127.0.0.1)."""
from __future__ import annotations

import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    out = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 0.5 * rank], dist, device="cpu")
    q.put((rank, out))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0] == res[1] == [2.0, 10.0, 0.5]


def test_max_over_ranks_single_process_is_identity():
    import bench
    assert bench.max_over_ranks([3.0, 4.0]) == [3.0, 4.0]
