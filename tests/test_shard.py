"""Multi-GPU binary splitting (piculator_b200/shard.py) on the CPU: the
range split, the pairwise merges up the tree and the NCCL-style exchange of
numbers, run over gloo ranks with the CPU checker as the arithmetic backend.
Rank 0's pi.txt text must equal the single-process computation's."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from piculator_b200.shard import bsr_tree, pi_distributed, shard_ranges


class OracleBackend:
    """The shard driver's backend interface on the CPU checker (numbers are
    (sign, exp, words) records; words travel as int32 CPU tensors)."""
    device = torch.device("cpu")

    def __init__(self):
        from oracle.ffi import Oracle
        self.o = Oracle()

    def bsr(self, a, b, p):
        return self.o.bsr(a, b, p)

    def mul(self, x, y, p):
        return self.o.mul(x, y, p)

    def add(self, x, y, p):
        return self.o.add(x, y, p)

    def mul_u32(self, x, s):
        return self.o.mul_u32(x, s)

    def div(self, x, y, p):
        return self.o.div(x, y, p)

    def invsqrt(self, s, p):
        return self.o.invsqrt(s, p)

    def empty(self):
        from oracle.ffi import BF
        return BF(True, 0, np.zeros(0, dtype=np.uint32))

    def pack(self, x):
        t = torch.from_numpy(x.words.astype(np.uint32).view(np.int32).copy()) if x.words.size else None
        return x.sign, x.exp, t

    def unpack(self, sign, exp, t):
        from oracle.ffi import BF
        w = t.numpy().view(np.uint32).copy() if t is not None else np.zeros(0, dtype=np.uint32)
        return BF(sign, exp, w)

    def to_hex(self, x, digits):
        # BigFloat::to_string_hex (BigFloat.cpp:95-106)
        w = x.words
        s = str(int(w[-1])) + "." + "".join(f"{int(v):08x}" for v in w[-2::-1][: (digits + 7) // 8])
        return s[: 2 + digits].encode()


def test_shard_ranges_follow_the_reference_split():
    assert shard_ranges(0, 10, 1) == [(0, 5), (5, 10)]
    assert shard_ranges(0, 11, 2) == [(0, 2), (2, 5), (5, 8), (8, 11)]
    r = shard_ranges(3, 1000, 5)
    assert len(r) == 32 and r[0][0] == 3 and r[-1][1] == 1000
    assert all(x[1] == y[0] for x, y in zip(r, r[1:]))
    with pytest.raises(ValueError):
        shard_ranges(0, 3, 2)


@pytest.mark.parametrize("depth", [1, 2, 3])
def test_bsr_tree_equals_single_recursion(depth):
    be = OracleBackend()
    _, p, terms = be.o.pi_sizes(20_000)
    P, Q, R = bsr_tree(be, 0, terms, p, depth)
    P1, Q1, R1 = be.o.bsr(0, terms, p)
    for x, y in ((P, P1), (Q, Q1), (R, R1)):
        assert x.sign == y.sign and x.exp == y.exp and np.array_equal(x.words, y.words)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, digits, q):
    import datetime
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    be = OracleBackend()
    text = pi_distributed(be, dist, digits, be.o.pi_sizes)
    q.put((rank, text))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3, 4, 6, 8])
def test_pi_over_gloo_ranks_equals_single_process(world):
    digits = 20_000
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, digits, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(res[r] is None for r in range(1, world))
    from oracle.ffi import Oracle
    assert res[0] == Oracle().pi_hex(digits)
