"""The FP64 three-prime product form (PIC_MUL_NTT3D): 56-bit pieces, three
primes below 2^47, butterflies and CRT in FP64 arithmetic.  Every product must
equal the oracle's, Python integers' and the integer form's words exactly."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.ffi import random_words

pytestmark = pytest.mark.gpu


def _int(w):
    return int.from_bytes(np.ascontiguousarray(w, dtype="<u4").tobytes(), "little")


@pytest.mark.parametrize("na,nb", [(1, 1), (1, 2), (2, 3), (7, 7), (31, 33), (64, 64), (100, 1), (1, 257),
                                   (255, 256), (1000, 1000), (1023, 2000), (2047, 2049), (4097, 3),
                                   (7, 7777)])
def test_products_vs_oracle(pic, oracle, na, nb):
    a = random_words(na * 7 + nb, na)
    b = random_words(nb * 13 + na, nb)
    assert np.array_equal(pic.mul_host(a, b, "ntt3d"), oracle.mul_words(a, b))


@pytest.mark.parametrize("n", [5000, 1 << 14, 40000, 1 << 17, 300001])
def test_products_vs_python_int(pic, n):
    a = random_words(n, n)
    b = random_words(n + 1, n - 3)
    assert _int(pic.mul_host(a, b, "ntt3d")) == _int(a) * _int(b)


def test_all_ones_max_carry_chain(pic):
    # (B^n - 1)^2: every coefficient at its largest, the longest carry chains
    for n in (3, 4097, 1 << 16, (1 << 18) + 5, 1 << 21):
        ones = np.full(n, 0xFFFFFFFF, dtype=np.uint32)
        z = pic.mul_host(ones, ones, "ntt3d")
        assert z[0] == 1 and np.all(z[1:n] == 0)
        assert z[n] == 0xFFFFFFFE and np.all(z[n + 1:] == 0xFFFFFFFF)


@pytest.mark.parametrize("na,nb", [(2200, 2200), (2201, 2199), (3000, 1300), (60000, 10000), (92000, 46000),
                                   (150000, 150000)])
def test_wrapped_and_plain_forms(pic, na, nb):
    a = random_words(na + 5, na)
    b = random_words(nb + 9, nb)
    want = _int(a) * _int(b)
    saved = pic.get_tuning(pic.TUNE_MUL_WRAP)
    try:
        for wrap in (1, 0):
            pic.set_tuning(pic.TUNE_MUL_WRAP, wrap)
            assert _int(pic.mul_host(a, b, "ntt3d")) == want, f"wrap={wrap}"
    finally:
        pic.set_tuning(pic.TUNE_MUL_WRAP, saved)


def test_squaring_same_pointer(pic, torch_cuda, oracle):
    torch = torch_cuda
    for n in (3000, 2200):
        a = random_words(77 + n, n)
        ta = torch.from_numpy(a.view(np.int32)).cuda()
        z = torch.zeros(2 * n, dtype=torch.int32, device="cuda")
        pic.mul_dev(z.data_ptr(), ta.data_ptr(), n, ta.data_ptr(), n, "ntt3d", torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert np.array_equal(z.cpu().numpy().view(np.uint32), oracle.mul_words(a, a))


@pytest.mark.parametrize("row_bits", [11, 12, 13])
def test_geometries_match_integer_form(pic, row_bits):
    """Every FP64 pass geometry (rows of 2^11 .. 2^13 points, radix-8 and
    radix-16 rounds) gives the integer form's words, for transform lengths
    2^14 .. 2^24, and Python integers where they are quick."""
    saved = {k: pic.get_ntt_geometry(k, pic.FORM_DBL) for k in range(14, 26)}
    try:
        for lg in (13, 16, 19, 22):
            n = 1 << lg
            a, b = random_words(lg + row_bits, n), random_words(lg + 2 * row_bits, n - 5)
            want = pic.mul_host(a, b, "ntt3")
            for rb in (3, 4):
                for k in range(14, 26):
                    pic.set_ntt_geometry(k, row_bits, saved[k][1], rb, pic.FORM_DBL)
                got = pic.mul_host(a, b, "ntt3d")
                assert np.array_equal(got, want), (lg, rb)
            if lg <= 16:
                assert _int(want) == _int(a) * _int(b)
    finally:
        for k, (r, lw, rb) in saved.items():
            pic.set_ntt_geometry(k, r, lw, rb, pic.FORM_DBL)


@pytest.mark.parametrize("lg", [22, 24])
def test_large_products_agree_with_integer_form(pic, lg):
    n = 1 << lg
    a, b = random_words(42, n), random_words(43, n)
    assert np.array_equal(pic.mul_host(a, b, "ntt3d"), pic.mul_host(a, b, "ntt3"))


def _pi_in_form(pic, digits, form):
    saved = pic.get_tuning(pic.TUNE_NTT_FORM)
    pic.set_tuning(pic.TUNE_NTT_FORM, form)
    try:
        return pic.pi_hex(digits, pic.PI_CHOSEN)
    finally:
        pic.set_tuning(pic.TUNE_NTT_FORM, saved)


@pytest.mark.parametrize("digits", [10_000, 100_000, 1_000_000, 3_141_593, 10_000_000, 27_182_818])
def test_pi_in_fp64_form_matches_reference(pic, golden, digits):
    """The whole computation (binary-splitting merges, Newton products) in the
    FP64 form: every hex digit equal to the reference's pi.txt."""
    import hashlib
    text, _ = _pi_in_form(pic, digits, pic.FORM_DBL)
    g = golden["pi"][str(digits)]
    assert len(text) == g["bytes"]
    assert hashlib.md5(text).hexdigest() == g["md5"]


@pytest.mark.slow
@pytest.mark.parametrize("digits", [100_000_000, 1_000_000_000])
def test_pi_in_fp64_form_large(pic, golden, digits):
    import hashlib
    text, _ = _pi_in_form(pic, digits, pic.FORM_DBL)
    assert hashlib.md5(text).hexdigest() == golden["pi"][str(digits)]["md5"]


@pytest.mark.parametrize("row_bits", [11, 12, 13])
def test_cols_bulk_kernel_matches_integer_form(pic, row_bits):
    """FP64 column passes through the persistent kernel fed by TMA bulk copies
    (PIC_TUNE_COLS_BULK): every column height 2^5 .. 2^9 it serves, tile widths
    2^3 .. 2^6, radix 8 and 16, with and without per-point pass tables, give
    the integer form's words."""
    saved = {k: pic.get_ntt_geometry(k, pic.FORM_DBL) for k in range(14, 26)}
    knobs = {pic.TUNE_COLS_BULK: pic.get_tuning(pic.TUNE_COLS_BULK),
             pic.TUNE_DBL_PASS_TABLES: pic.get_tuning(pic.TUNE_DBL_PASS_TABLES)}
    try:
        for lg, bits in ((16, 12), (19, 10), (22, 11)):
            pic.set_tuning(pic.TUNE_COLS_BULK, bits)
            n = 1 << lg
            a, b = random_words(lg + 3 * row_bits, n), random_words(lg + 5 * row_bits, n - 7)
            want = pic.mul_host(a, b, "ntt3")
            for lw, rb, tables in ((0, 3, 24), (3, 4, 24), (6, 3, 0), (4, 3, 20)):
                pic.set_tuning(pic.TUNE_DBL_PASS_TABLES, tables)
                for k in range(14, 26):
                    pic.set_ntt_geometry(k, row_bits, lw, rb, pic.FORM_DBL)
                assert np.array_equal(pic.mul_host(a, b, "ntt3d"), want), (lg, lw, rb, tables)
    finally:
        for k, (r, lw, rb) in saved.items():
            pic.set_ntt_geometry(k, r, lw, rb, pic.FORM_DBL)
        for k, v in knobs.items():
            pic.set_tuning(k, v)


@pytest.mark.parametrize("digits", [1_000_000, 10_000_000, 27_182_818])
def test_pi_with_cols_bulk_kernel(pic, golden, digits):
    import hashlib
    saved = pic.get_tuning(pic.TUNE_COLS_BULK)
    pic.set_tuning(pic.TUNE_COLS_BULK, 10)
    try:
        text, _ = _pi_in_form(pic, digits, pic.FORM_DBL)
    finally:
        pic.set_tuning(pic.TUNE_COLS_BULK, saved)
    assert hashlib.md5(text).hexdigest() == golden["pi"][str(digits)]["md5"]


@pytest.mark.parametrize("digits", [1_000_000, 10_000_000, 27_182_818])
def test_pi_in_chosen_form(pic, golden, digits):
    """Form chosen per product and merge level (PIC_TUNE_NTT_FORM 2): levels
    and products of both forms in one computation, the reference's digits."""
    import hashlib
    text, _ = _pi_in_form(pic, digits, pic.FORM_CHOSEN)
    assert hashlib.md5(text).hexdigest() == golden["pi"][str(digits)]["md5"]


@pytest.mark.parametrize("n", [1000, 5000, 1 << 14, 40000, 1 << 17, 300001])
def test_auto_products_in_chosen_form(pic, n):
    a = random_words(n + 17, n)
    b = random_words(n + 19, n - 3)
    saved = pic.get_tuning(pic.TUNE_NTT_FORM)
    pic.set_tuning(pic.TUNE_NTT_FORM, pic.FORM_CHOSEN)
    try:
        z = pic.mul_host(a, b, "auto")
    finally:
        pic.set_tuning(pic.TUNE_NTT_FORM, saved)
    assert _int(z) == _int(a) * _int(b)
