"""The multi-GPU binary splitting's device side on one GPU: its range split
and merges (all subtrees in one process, merged as the ranks would merge
them) give the same P, Q, R as the single batched splitting; numbers survive
the device-to-device pack / unpack used for the NCCL exchange; and the
distributed driver with one rank writes the reference's pi.txt."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


class Solo:
    def get_rank(self):
        return 0

    def get_world_size(self):
        return 1


@pytest.mark.parametrize("depth", [1, 3])
def test_bsr_tree_on_device_equals_batched(pic, depth):
    from piculator_b200.shard import DeviceBackend, bsr_tree
    be = DeviceBackend()
    _, p, terms = pic.pi_sizes(1_000_000)
    got = bsr_tree(be, 0, terms, p, depth)
    want = pic.bsr(0, terms, p)
    for x, y in zip(got, want):
        a, b = x.to_bf(), y.to_bf()
        assert a.sign == b.sign and a.exp == b.exp and np.array_equal(a.words, b.words)


def test_pack_unpack_round_trip(pic):
    from piculator_b200.shard import DeviceBackend
    be = DeviceBackend()
    w = (np.arange(1, 100001, dtype=np.uint64) * 2654435761 % (1 << 32)).astype(np.uint32)
    x = pic.DeviceBigFloat.from_words(False, -7, w)
    sign, exp, t = be.pack(x)
    y = be.unpack(sign, exp, t)
    b = y.to_bf()
    assert (b.sign, b.exp) == (False, -7) and np.array_equal(b.words, w)
    e = be.unpack(True, 0, None).to_bf()
    assert e.words.size == 0


def test_pi_distributed_single_rank(pic, golden):
    from piculator_b200.shard import DeviceBackend, pi_distributed
    text = pi_distributed(DeviceBackend(), Solo(), 1_000_000, pic.pi_sizes)
    assert hashlib.md5(text).hexdigest() == golden["pi"]["1000000"]["md5"]
