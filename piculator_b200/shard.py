"""Multi-GPU binary splitting (one process per GPU, torch.distributed).

The reference forks Pi_BSR into two threads at every node whose range holds
at least 1000 terms (PI.h:93-108); the subtrees are independent until their
parent merges them (PI.h:110-112).  Across GPUs the same split is taken
log2(G) levels deep: rank r evaluates the r-th range at that depth on its own
GPU with the batched binary splitting, then the ranks merge pairwise up the
tree -- rank r + s sends its P, Q, R to rank r, which forms
P = P0 Q1 + P1 R0, Q = Q0 Q1, R = R0 R1 at precision p exactly as PI.h:110-112
-- so rank 0 ends with the reference's P, Q (R of the root is never used by
Pi(), PI.h:179-199, and is not formed).  The inverse square root of 10005
(PI.h:194) does not depend on the series: rank 1 computes it while rank 0
runs the top merges and the division, then sends it over.

Numbers move between GPUs as (sign, exponent, length) plus their 32-bit
words, device to device (pic_bf_to_device / pic_bf_from_device and NCCL
send/recv); every rank takes the same point-to-point steps in the same order.

The driver is written against a small backend interface (bsr, mul, add,
mul_u32, div, invsqrt, pack, unpack, to_hex) so the same merge and exchange
logic runs on the GPUs (DeviceBackend) and, in the tests, on the CPU checker
over gloo ranks.  G is the largest power of two not above the world size;
ranks beyond it stay idle.
"""
from __future__ import annotations

from typing import Optional


def shard_ranges(a: int, b: int, depth: int) -> list[tuple[int, int]]:
    """The 2^depth node ranges of the reference's recursion at `depth`, left
    to right: every split at m = (a + b) / 2 (PI.h:90)."""
    out = [(a, b)]
    for _ in range(depth):
        nxt = []
        for x, y in out:
            if y - x < 2:
                raise ValueError(f"range [{x}, {y}) has no split at depth {depth}")
            m = (x + y) // 2
            nxt += [(x, m), (m, y)]
        out = nxt
    return out


def merge(be, left, right, p: int, need_r: bool = True):
    """PI.h:110-112 on two adjacent nodes (left = [a, m), right = [m, b))."""
    P0, Q0, R0 = left
    P1, Q1, R1 = right
    P = be.add(be.mul(P0, Q1, p), be.mul(P1, R0, p), p)
    Q = be.mul(Q0, Q1, p)
    R = be.mul(R0, R1, p) if need_r else None
    return P, Q, R


def bsr_tree(be, a: int, b: int, p: int, depth: int, need_root_r: bool = True):
    """All 2^depth subtrees in this process, merged level by level: the
    multi-GPU schedule run on one device (its merges and ranges are the
    distributed ones)."""
    nodes = [be.bsr(x, y, p) for x, y in shard_ranges(a, b, depth)]
    while len(nodes) > 1:
        last = len(nodes) == 2
        nodes = [merge(be, nodes[i], nodes[i + 1], p, need_r=need_root_r or not last)
                 for i in range(0, len(nodes), 2)]
    return nodes[0]


def _send(be, dist, x, dst: int) -> None:
    import torch
    sign, exp, words = be.pack(x)
    n = int(words.numel()) if words is not None else 0
    meta = torch.tensor([int(sign), int(exp), n], dtype=torch.int64, device=be.device)
    dist.send(meta, dst)
    if n:
        dist.send(words, dst)


def _recv(be, dist, src: int):
    import torch
    meta = torch.empty(3, dtype=torch.int64, device=be.device)
    dist.recv(meta, src)
    sign, exp, n = (int(v) for v in meta.tolist())
    words = None
    if n:
        words = torch.empty(n, dtype=torch.int32, device=be.device)
        dist.recv(words, src)
    return be.unpack(bool(sign), exp, words)


def bsr_distributed(be, dist, a: int, b: int, p: int, need_root_r: bool = False):
    """Binary splitting of [a, b) over the ranks; rank 0 returns (P, Q, R),
    the others None once they have handed their node up the tree."""
    rank, world = dist.get_rank(), dist.get_world_size()
    depth = world.bit_length() - 1
    n = 1 << depth
    if rank >= n:
        return None
    node = be.bsr(*shard_ranges(a, b, depth)[rank], p)
    step = 1
    while step < n:
        if rank % (2 * step) == 0:
            right = tuple(_recv(be, dist, rank + step) for _ in range(3))
            node = merge(be, node, right, p, need_r=need_root_r or 2 * step < n)
        else:
            for x in node:
                _send(be, dist, x if x is not None else be.empty(), rank - step)
            return None
        step *= 2
    return node


def pi_distributed(be, dist, digits: int, sizes) -> Optional[bytes]:
    """Pi() (PI.h:138-212) over the ranks; rank 0 returns the pi.txt text."""
    hexd, p, terms = sizes(digits)
    rank, world = dist.get_rank(), dist.get_world_size()
    node = bsr_distributed(be, dist, 0, terms, p)
    if rank == 1 and world >= 2:
        _send(be, dist, be.invsqrt(10005, p), 0)  # PI.h:194, off rank 0's path
        return None
    if rank != 0:
        return None
    P, Q, _ = node
    P = be.add(be.mul_u32(Q, 13591409), P, p)  # PI.h:180
    Q = be.mul_u32(Q, 4270934400)               # PI.h:181
    P = be.div(Q, P, p)                         # PI.h:189
    Q = _recv(be, dist, 1) if world >= 2 else be.invsqrt(10005, p)
    P = be.mul(P, Q, p)                         # PI.h:199
    return be.to_hex(P, hexd)                   # PI.h:204


class DeviceBackend:
    """The backend on this process's GPU (pic_bf handles; words cross GPUs as
    int32 CUDA tensors through NCCL)."""

    def __init__(self):
        import torch

        import piculator_b200 as P
        self.P = P
        self.torch = torch
        self.device = torch.device("cuda", torch.cuda.current_device())

    def _stream(self):
        return self.torch.cuda.current_stream().cuda_stream or None

    def bsr(self, a, b, p):
        return self.P.bsr(a, b, p, self.P.PI_CHOSEN)

    def mul(self, x, y, p):
        return x.mul(y, p)

    def add(self, x, y, p):
        return x.add(y, p)

    def mul_u32(self, x, s):
        return x.mul_u32(s)

    def div(self, x, y, p):
        return x.div(y, p)

    def invsqrt(self, s, p):
        return self.P.DeviceBigFloat.invsqrt(s, p)

    def empty(self):
        import numpy as np
        return self.P.DeviceBigFloat.from_words(True, 0, np.zeros(0, dtype=np.uint32))

    def pack(self, x):
        sign, exp, n = x.info()
        if n == 0:
            return sign, exp, None
        t = self.torch.empty(n, dtype=self.torch.int32, device=self.device)
        self.P.check(self.P.lib().pic_bf_to_device(x.h, t.data_ptr(), n, self._stream()))
        return sign, exp, t

    def unpack(self, sign, exp, words):
        import ctypes as C
        out = C.c_void_p()
        n = 0 if words is None else int(words.numel())
        ptr = words.data_ptr() if n else None
        self.P.check(self.P.lib().pic_bf_from_device(C.byref(out), int(sign), int(exp), ptr, n, self._stream()))
        return self.P.DeviceBigFloat(out.value)

    def to_hex(self, x, digits):
        return x.to_hex(digits)
