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


@pytest.mark.parametrize("n", [2, 3, 8])
def test_bench_gpus_flag_launches_n_replicas(n):
    """`bench.py --gpus N` outside torchrun re-launches itself as N ranks
    (torch.distributed.run on 127.0.0.1); with the launcher's self-test arm
    (gloo, no GPU) rank 0 prints one line whose n_gpus is N."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--gpus", str(n), "--impl",
                        "replica-check", "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, timeout=240, env=env, cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    assert lines[0]["n_gpus"] == n and lines[0]["per_rank_max_of"] == n


def test_bench_rejects_rank_count_mismatch():
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--gpus", "2", "--impl",
                        "replica-check"], capture_output=True, text=True, timeout=120, env=env, cwd=root)
    assert r.returncode != 0 and "ranks were launched" in r.stderr


def test_reference_arm_under_two_ranks_prints_one_line():
    """`bench.py --gpus 2 --impl reference`: rank 0 alone times the reference
    program and prints the line; the other rank exits 0 without work."""
    import json
    import subprocess
    import sys

    from oracle.ffi import REF_PI, REF_SO
    if not (os.path.exists(REF_PI) and os.path.exists(REF_SO)):
        pytest.skip("oracle/_ref not built (the reference sources are not in this checkout)")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = {k: v for k, v in os.environ.items() if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK")}
    r = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--gpus", "2", "--impl", "reference",
                        "--steps", "1", "--warmup", "1", "--digits", "1000000", "--ref-sample", "10000",
                        "--ref-calibration", "100000"], capture_output=True, text=True, timeout=600, env=env,
                       cwd=root)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1 and lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2
