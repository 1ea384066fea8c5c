"""pic_mul_batch: many uneven products per call (persistent schoolbook +
binned three-prime NTT, replayed from a captured CUDA graph), checked word for
word against the single-product entry point and the oracle, and on the full
8192-product workload by mod-prime fingerprints."""
from __future__ import annotations

import math

import numpy as np
import pytest

from oracle.ffi import random_words, splitmix64_np

pytestmark = pytest.mark.gpu

Q = (2 ** 61 - 1, 1000000007)


def log_uniform_sizes(seed: int, count: int, top: int) -> list[int]:
    """floor(exp(U(0, ln top))) clamped to [1, top], U from splitmix64(seed)."""
    u = (splitmix64_np(seed, count) >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    return [max(1, min(top, int(math.exp(x * math.log(top))))) for x in u]


def _setup(torch, sizes_a, sizes_b, seed):
    ops = []
    for i, (na, nb) in enumerate(zip(sizes_a, sizes_b)):
        a = random_words(seed + 2 * i, na)
        b = random_words(seed + 2 * i + 1, nb)
        ops.append((a, b))
    flat_a = np.concatenate([a for a, _ in ops])
    flat_b = np.concatenate([b for _, b in ops])
    ta = torch.from_numpy(flat_a.view(np.int32)).cuda()
    tb = torch.from_numpy(flat_b.view(np.int32)).cuda()
    tz = torch.zeros(int(flat_a.size + flat_b.size), dtype=torch.int32, device="cuda")
    descs, oa, ob, oz = [], 0, 0, 0
    for a, b in ops:
        descs.append((tz.data_ptr() + 4 * oz, ta.data_ptr() + 4 * oa, a.size, tb.data_ptr() + 4 * ob, b.size))
        oa += a.size
        ob += b.size
        oz += a.size + b.size
    return ops, descs, (ta, tb, tz)


def _outputs(tz, ops):
    z = tz.cpu().numpy().view(np.uint32)
    out, o = [], 0
    for a, b in ops:
        out.append(z[o:o + a.size + b.size])
        o += a.size + b.size
    return out


def _int(w):
    return int.from_bytes(np.ascontiguousarray(w, dtype="<u4").tobytes(), "little")


@pytest.mark.parametrize("graphs", [1, 0])
def test_batch_equals_single_products(pic, torch_cuda, graphs):
    torch = torch_cuda
    sizes = log_uniform_sizes(11, 300, 20000)
    sizes_b = log_uniform_sizes(12, 300, 20000)
    pic.set_tuning(pic.TUNE_BATCH_GRAPHS, graphs)
    try:
        ops, descs, (ta, tb, tz) = _setup(torch, sizes, sizes_b, 100)
        s = torch.cuda.current_stream().cuda_stream
        pic.mul_batch_dev(descs, "auto", s)
        torch.cuda.synchronize()
        got = _outputs(tz, ops)
        for (z_ptr, a_ptr, na, b_ptr, nb), g in zip(descs, got):
            ref = torch.zeros(na + nb, dtype=torch.int32, device="cuda")
            pic.mul_dev(ref.data_ptr(), a_ptr, na, b_ptr, nb, "ntt3", s)
            torch.cuda.synchronize()
            assert np.array_equal(ref.cpu().numpy().view(np.uint32), g)
    finally:
        pic.set_tuning(pic.TUNE_BATCH_GRAPHS, 1)


def test_batch_config3_workload_and_graph_replay(pic, torch_cuda, oracle):
    """8192 products per call, operand sizes log-uniform in 1..8192 limbs
    (splitmix64 seed 7); the second call has the same sizes and new operands,
    so it runs from the captured graph."""
    torch = torch_cuda
    sizes = log_uniform_sizes(7, 2 * 8192, 8192)
    sa, sb = sizes[0::2], sizes[1::2]
    s = torch.cuda.current_stream().cuda_stream
    for call, seed in enumerate((1000, 5000000)):
        ops, descs, (ta, tb, tz) = _setup(torch, sa, sb, seed)
        pic.mul_batch_dev(descs, "auto", s)
        torch.cuda.synchronize()
        got = _outputs(tz, ops)
        for (a, b), z in zip(ops, got):
            ia, ib, iz = _int(a), _int(b), _int(z)
            for q in Q:
                assert iz % q == (ia % q) * (ib % q) % q
        for i in range(0, 8192, 257):  # exact words for a sample
            a, b = ops[i]
            assert np.array_equal(got[i], oracle.mul_words(a, b)), (call, i)
