"""Whole products (pic_mul / pic_mul_host / pic_mul_batch) vs the oracle,
Python integers and the reference goldens."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from oracle.ffi import random_words

pytestmark = pytest.mark.gpu

MODES = ["school", "ntt_ref", "ntt3", "ntt3d", "fft", "auto"]


def _md5(w):
    return hashlib.md5(np.ascontiguousarray(w, dtype="<u4").tobytes()).hexdigest()


def _int(w):
    return int.from_bytes(np.ascontiguousarray(w, dtype="<u4").tobytes(), "little")


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("na,nb", [(1, 1), (1, 2), (2, 3), (7, 7), (31, 33), (64, 64), (100, 1),
                                   (1, 257), (255, 256), (1000, 1000), (1023, 2000), (2047, 2049)])
def test_products_vs_oracle(pic, oracle, mode, na, nb):
    a = random_words(na * 7 + nb, na)
    b = random_words(nb * 13 + na, nb)
    z = pic.mul_host(a, b, mode)
    assert np.array_equal(z, oracle.mul_words(a, b))


@pytest.mark.parametrize("mode", ["ntt_ref", "ntt3", "fft", "auto"])
@pytest.mark.parametrize("n", [5000, 1 << 14, 40000, 1 << 17])
def test_products_vs_python_int(pic, mode, n):
    a = random_words(n, n)
    b = random_words(n + 1, n - 3)
    z = pic.mul_host(a, b, mode)
    assert _int(z) == _int(a) * _int(b)


@pytest.mark.parametrize("mode", MODES)
def test_edge_products_golden(pic, golden, mode):
    for rec in golden["products"]["edge"]:
        n = rec["n"]
        ones = np.full(n, 0xFFFFFFFF, dtype=np.uint32)
        if rec["kind"] == "ones":
            a, b = ones, ones
        else:
            a = np.zeros(n, dtype=np.uint32)
            a[0] = 1
            a[-1] = 1
            b = ones
        z = pic.mul_host(a, b, mode)
        L = z.size - (1 if z[-1] == 0 else 0)
        assert L == rec["L"] and _md5(z[:L]) == rec["md5"]


@pytest.mark.parametrize("lg", [12, 16, 20])
@pytest.mark.parametrize("mode", ["ntt_ref", "ntt3", "ntt3d", "fft", "auto"])
def test_isolated_products_golden(pic, golden, lg, mode):
    rec = [r for r in golden["products"]["isolated"] if r["log2n"] == lg][0]
    n = 1 << lg
    z = pic.mul_host(random_words(42, n), random_words(43, n), mode)
    L = z.size - (1 if z[-1] == 0 else 0)
    assert L == rec["L"] and _md5(z[:L]) == rec["md5"]


@pytest.fixture(scope="module")
def big_operands():
    cache = {}

    def get(lg):
        if lg not in cache:
            cache.clear()
            n = 1 << lg
            cache[lg] = (random_words(42, n), random_words(43, n))
        return cache[lg]
    return get


# The isolated-multiply workload at its two largest sizes: 2^24 and 2^27
# words per operand, the reference's NTT at k = 27 and k = 30
# (BigFloat.cpp:380-441).  The fixture holds the md5 of the reference's own
# product words.  The FP64 FFT has no proven piece width at these lengths.
@pytest.mark.parametrize("lg", [24, 27])
@pytest.mark.parametrize("mode", ["ntt3", "ntt3d", "ntt_ref", "auto"])
def test_isolated_products_golden_large(pic, golden, big_operands, lg, mode):
    rec = [r for r in golden["products"]["isolated"] if r["log2n"] == lg][0]
    a, b = big_operands(lg)
    z = pic.mul_host(a, b, mode)
    L = z.size - (1 if z[-1] == 0 else 0)
    assert L == rec["L"] and int(z[L - 1]) == rec["top"]
    assert _md5(z[:L]) == rec["md5"]


def test_fft_beyond_proven_bound_is_refused(pic):
    n = 1 << 24
    a = np.ones(n, dtype=np.uint32)
    with pytest.raises(pic.PicError) as e:
        pic.mul_host(a, a, "fft")
    assert e.value.status == pic.ERR_LENGTH


@pytest.mark.parametrize("lg", [22, 24])
def test_large_products_fingerprint(pic, lg):
    """Mod-prime fingerprints where Python-int products would be slow:
    z mod q == (a mod q)(b mod q) mod q for several 61-bit primes, and the
    NTT forms agree word for word."""
    n = 1 << lg
    a, b = random_words(42, n), random_words(43, n)
    z3 = pic.mul_host(a, b, "ntt3")
    zr = pic.mul_host(a, b, "ntt_ref")
    assert np.array_equal(z3, zr)
    ia, ib, iz = _int(a), _int(b), _int(z3)
    for q in (2 ** 61 - 1, 2305843009213693921, 1000000007):
        assert iz % q == (ia % q) * (ib % q) % q


def test_all_ones_max_carry_chain(pic):
    # (B^n - 1)^2 = B^2n - 2 B^n + 1: the longest possible carry chains
    for n in (3, 4097, 1 << 16, (1 << 18) + 5):
        ones = np.full(n, 0xFFFFFFFF, dtype=np.uint32)
        for mode in ("ntt3", "ntt_ref", "fft"):
            z = pic.mul_host(ones, ones, mode)
            assert z[0] == 1 and np.all(z[1:n] == 0)
            assert z[n] == 0xFFFFFFFE and np.all(z[n + 1:] == 0xFFFFFFFF)


# Sizes whose coefficient count just exceeds a power of two: the three-prime
# product takes the wrapped form (main transform at the smaller power plus a
# tail product), for equal, unequal and odd operand lengths.
@pytest.mark.parametrize("na,nb", [(2200, 2200), (2201, 2199), (3000, 1300), (60000, 10000), (92000, 46000)])
def test_wrapped_products(pic, na, nb):
    a = random_words(na + 5, na)
    b = random_words(nb + 9, nb)
    want = _int(a) * _int(b)
    saved = pic.get_tuning(pic.TUNE_MUL_WRAP)
    try:
        for wrap in (1, 0):
            pic.set_tuning(pic.TUNE_MUL_WRAP, wrap)
            z = pic.mul_host(a, b, "ntt3")
            assert _int(z) == want, f"wrap={wrap}"
    finally:
        pic.set_tuning(pic.TUNE_MUL_WRAP, saved)


def test_wrapped_square_same_pointer(pic, torch_cuda):
    torch = torch_cuda
    n = 2200
    a = random_words(91, n)
    ta = torch.from_numpy(a.view(np.int32)).cuda()
    z = torch.zeros(2 * n, dtype=torch.int32, device="cuda")
    pic.mul_dev(z.data_ptr(), ta.data_ptr(), n, ta.data_ptr(), n, "ntt3", torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert _int(z.cpu().numpy().view(np.uint32)) == _int(a) ** 2


def test_squaring_same_pointer(pic, torch_cuda, oracle):
    torch = torch_cuda
    a = random_words(77, 3000)
    ta = torch.from_numpy(a.view(np.int32)).cuda()
    z = torch.zeros(6000, dtype=torch.int32, device="cuda")
    for mode in ("ntt3", "ntt_ref", "fft", "school"):
        z.zero_()
        pic.mul_dev(z.data_ptr(), ta.data_ptr(), 3000, ta.data_ptr(), 3000, mode,
                    torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert np.array_equal(z.cpu().numpy().view(np.uint32), oracle.mul_words(a, a))


def test_mul_batch_uneven(pic, torch_cuda, oracle):
    torch = torch_cuda
    rng = np.random.default_rng(7)
    sizes = [(int(x), int(y)) for x, y in rng.integers(1, 3000, (40, 2))]
    ops, descs = [], []
    for i, (na, nb) in enumerate(sizes):
        a, b = random_words(2 * i, na), random_words(2 * i + 1, nb)
        ta = torch.from_numpy(a.view(np.int32)).cuda()
        tb = torch.from_numpy(b.view(np.int32)).cuda()
        tz = torch.zeros(na + nb, dtype=torch.int32, device="cuda")
        ops.append((a, b, ta, tb, tz))
        descs.append((tz.data_ptr(), ta.data_ptr(), na, tb.data_ptr(), nb))
    pic.mul_batch_dev(descs, "auto", torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    for a, b, _, _, tz in ops:
        assert np.array_equal(tz.cpu().numpy().view(np.uint32), oracle.mul_words(a, b))


def test_fft_error_is_logged(pic):
    a, b = random_words(1, 1 << 15), random_words(2, 1 << 15)
    n0 = pic.lib().pic_fft_recompute_count()
    pic.mul_host(a, b, "fft")
    e = pic.lib().pic_fft_last_max_err()
    assert 0.0 < e < 0.25
    assert pic.lib().pic_fft_recompute_count() == n0


@pytest.mark.parametrize("n", [1 << 12, 1 << 15, 100000])
def test_fft_recompute_past_threshold(pic, n):
    """With the acceptance threshold lowered below the products' rounding
    distance, every FFT product takes the NTT recompute branch: the words are
    still exact and the recompute counter moves by one per product."""
    L = pic.lib()
    a, b = random_words(3 * n, n), random_words(3 * n + 1, n - 7)
    want = _int(a) * _int(b)
    saved = pic.get_tuning(pic.TUNE_FFT_ACCEPT_PPM)
    assert saved == 250000
    try:
        pic.set_tuning(pic.TUNE_FFT_ACCEPT_PPM, 0)
        n0 = L.pic_fft_recompute_count()
        z = pic.mul_host(a, b, "fft")
        assert L.pic_fft_last_max_err() > 0.0
        assert L.pic_fft_recompute_count() == n0 + 1
        assert _int(z) == want
    finally:
        pic.set_tuning(pic.TUNE_FFT_ACCEPT_PPM, saved)
    n1 = L.pic_fft_recompute_count()
    assert _int(pic.mul_host(a, b, "fft")) == want
    assert L.pic_fft_recompute_count() == n1


@pytest.mark.parametrize("row_bits", [11, 12, 13])
def test_radix16_row_passes(pic, row_bits):
    """Passes with radix-16 register rounds (geometry radix_log2 4: rows of
    2^11 .. 2^13 points, columns of 2^8 .. 2^11 rows) give the same words as
    radix-8 rounds, for lengths 2^14 .. 2^23, and Python integers where they
    are quick (2^14, 2^17)."""
    saved = {k: pic.get_ntt_geometry(k) for k in range(14, 25)}
    try:
        for lg in (14, 17, 20, 23):
            n = 1 << lg  # n words -> about n pieces -> length 2^lg
            a, b = random_words(lg + row_bits, n), random_words(lg + 2 * row_bits, n - 5)
            got = {}
            for rb in (3, 4):
                for k in range(14, 25):
                    pic.set_ntt_geometry(k, row_bits, saved[k][1], rb)
                got[rb] = pic.mul_host(a, b, "ntt3")
            assert np.array_equal(got[3], got[4]), lg
            if lg <= 17:
                assert _int(got[4]) == _int(a) * _int(b), lg
    finally:
        for k, (r, lw, rb) in saved.items():
            pic.set_ntt_geometry(k, r, lw, rb)
