"""BigFloat semantics (truncation windows, carries, Newton steps) on the GPU
vs the reference goldens and the oracle."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.ffi import BF

pytestmark = pytest.mark.gpu


def _bf(rec):
    return BF(bool(rec[0]), int(rec[1]), np.array(rec[2], dtype=np.uint32))


def _same(dev, want: BF) -> bool:
    got = dev.to_bf()
    return (got.sign == want.sign and got.exp == want.exp and got.words.size == want.words.size
            and np.array_equal(got.words, want.words))


@pytest.mark.parametrize("mode", ["auto", "ntt_ref", "ntt3"])
def test_golden_ops(pic, golden, mode):
    D = pic.DeviceBigFloat
    for rec in golden["bigfloat"]["ops"]:
        a, b, p = D.from_bf(_bf(rec["a"])), D.from_bf(_bf(rec["b"])), rec["p"]
        assert _same(a.add(b, p), _bf(rec["add"]))
        assert _same(a.sub(b, p), _bf(rec["sub"]))
        assert _same(a.mul(b, p, mode), _bf(rec["mul"]))
        assert _same(a.rcp(p, mode), _bf(rec["rcp"]))
        assert _same(a.div(b, p, mode), _bf(rec["div"]))
        assert _same(a.mul_u32(rec["mul_u32"][0]), _bf(rec["mul_u32"][1:]))


def test_golden_invsqrt_and_carry_loss(pic, golden):
    D = pic.DeviceBigFloat
    for rec in golden["bigfloat"]["invsqrt"]:
        assert _same(D.invsqrt(rec["x"], rec["p"]), _bf(rec["z"]))
    c = golden["bigfloat"]["carry_loss"]
    assert _same(D.from_bf(_bf(c["a"])).add(D.from_bf(_bf(c["b"])), c["p"]), _bf(c["add"]))


def test_random_ops_vs_oracle(pic, oracle):
    D = pic.DeviceBigFloat
    rng = np.random.default_rng(11)
    for _ in range(60):
        na, nb = (int(v) for v in rng.integers(1, 3000, 2))
        a = rng.integers(0, 2 ** 32, na, dtype=np.uint64).astype(np.uint32)
        b = rng.integers(0, 2 ** 32, nb, dtype=np.uint64).astype(np.uint32)
        a[-1] |= 1
        b[-1] |= 1
        A = BF(bool(rng.integers(2)), int(rng.integers(-50, 50)), a)
        B = BF(bool(rng.integers(2)), int(rng.integers(-50, 50)), b)
        p = int(rng.integers(0, 2500))
        dA, dB = D.from_bf(A), D.from_bf(B)
        assert _same(dA.add(dB, p), oracle.add(A, B, p))
        assert _same(dA.sub(dB, p), oracle.sub(A, B, p))
        assert _same(dA.mul(dB, p), oracle.mul(A, B, p))
        assert dA.ucmp(dB) == oracle.ucmp(A, B)


def test_equal_magnitudes_subtract_to_zero(pic):
    D = pic.DeviceBigFloat
    w = np.array([5, 0xFFFFFFFF, 7], dtype=np.uint32)
    a, b = D.from_words(True, 3, w), D.from_words(True, 3, w)
    z = a.sub(b).to_bf()
    assert z.sign and z.exp == 0 and z.words.size == 0


def test_long_carry_and_borrow_chains(pic, oracle):
    D = pic.DeviceBigFloat
    n = 50000
    ones = BF(True, 0, np.full(n, 0xFFFFFFFF, dtype=np.uint32))
    one = BF(True, 0, np.array([1], dtype=np.uint32))
    big = BF(True, 0, np.concatenate([np.zeros(n, dtype=np.uint32), np.array([1], dtype=np.uint32)]))
    assert _same(D.from_bf(ones).add(D.from_bf(one)), oracle.add(ones, one))
    assert _same(D.from_bf(big).sub(D.from_bf(one)), oracle.sub(big, one))
    assert _same(D.from_bf(ones).mul_u32(0xFFFFFFFF), oracle.mul_u32(ones, 0xFFFFFFFF))


def test_divide_by_zero_status(pic):
    D = pic.DeviceBigFloat
    z = D.from_words(True, 0, np.zeros(0, dtype=np.uint32))
    with pytest.raises(pic.PicError) as e:
        z.rcp(10)
    assert e.value.status == pic.ERR_DIVIDE_BY_ZERO
    with pytest.raises(pic.PicError) as e:
        D.invsqrt(0, 10)
    assert e.value.status == pic.ERR_DIVIDE_BY_ZERO


def test_to_hex_matches_reference_format(pic, oracle):
    D = pic.DeviceBigFloat
    w = np.array([0x89abcdef, 0x01234567, 0xdeadbeef, 3], dtype=np.uint32)
    assert D.from_words(True, -3, w).to_hex(20) == b"3.deadbeef0123456789ab"


def test_transform_operands(pic, oracle):
    """Transform.h: forward once, multiply pointwise, metadata combined."""
    D = pic.DeviceBigFloat
    a = BF(False, 2, np.array([1, 2, 3, 0x80000000], dtype=np.uint32))
    b = BF(True, -1, np.array([7, 0xFFFFFFFF, 9], dtype=np.uint32))
    ta = pic.Transform(D.from_bf(a), 0, 4)
    tb = pic.Transform(D.from_bf(b), 0, 4)
    ta.mul(tb)
    z = ta.to_bigfloat()
    assert _same(z, oracle.mul(a, b, 0))
