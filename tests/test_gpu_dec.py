"""Decimal output (BigFloat::to_string_dec, BigFloat.cpp:83-94) on the GPU:
the reference program's own text for seeded numbers, edge cases and Pi()'s
number up to 10^6 digits; an exact check against Python integers at 2^21
words; and prefix consistency (a truncated expansion is a prefix of a longer
one) for pi up to 10^8 digits."""
from __future__ import annotations

import hashlib
import sys

import numpy as np
import pytest

from oracle.ffi import random_words

pytestmark = pytest.mark.gpu


def _md5(b: bytes) -> str:
    return hashlib.md5(b).hexdigest()


def test_numbers_match_reference(pic, golden):
    for i, rec in enumerate(golden["dec"]["numbers"]):
        w = random_words(rec["seed"], rec["L"])
        if rec["top_mod7"]:
            w[-1] = (w[-1] % 7) + 1
        x = pic.DeviceBigFloat.from_words(True, -rec["L"] + 1, w)
        text = x.to_dec(rec["digits"])
        assert len(text) == rec["len"], rec
        if "text" in rec:
            assert text.decode() == rec["text"], rec
        assert _md5(text) == rec["md5"], rec


def test_edge_numbers_match_reference(pic, golden):
    cases = {"ones": np.full(300, 0xFFFFFFFF, dtype=np.uint32),
             "zeros_below_top": np.array([0] * 299 + [3], dtype=np.uint32),
             "single_low_bit": np.array([1] + [0] * 298 + [3], dtype=np.uint32)}
    for rec in golden["dec"]["edge"]:
        x = pic.DeviceBigFloat.from_words(True, 0, cases[rec["kind"]])
        text = x.to_dec(rec["digits"])
        assert _md5(text) == rec["md5"] and text[-60:].decode() == rec["tail"], rec["kind"]


def _pi_bf(pic, digits):
    import ctypes as C
    h = C.c_void_p()
    st = pic.PiStats()
    pic.check(pic.lib().pic_pi_compute(digits, pic.PI_CHOSEN, C.byref(h), C.byref(st)))
    return pic.DeviceBigFloat(h.value)


@pytest.mark.parametrize("digits", [10_000, 100_000, 1_000_000])
def test_pi_decimal_matches_reference(pic, golden, digits):
    text = _pi_bf(pic, digits).to_dec(digits)
    g = golden["dec"]["pi"][str(digits)]
    assert len(text) == g["len"] and text[:80].decode() == g["head"]
    assert text[-80:].decode() == g["tail"]
    assert _md5(text) == g["md5"]


def test_exact_against_python_integers(pic):
    """N = floor(M 10^D / 2^B) for a 2^18-word fraction, D = 1,500,003."""
    sys.set_int_max_str_digits(0)
    L = (1 << 18) + 1
    w = random_words(99, L)
    w[-1] = 3
    digits = 1_500_003
    text = pic.DeviceBigFloat.from_words(True, 0, w).to_dec(digits)
    M = int.from_bytes(w[:-1].astype("<u4").tobytes(), "little")
    D = 9 * ((digits + 8) // 9)
    N = (M * 10 ** D) >> (32 * (L - 1))
    want = ("3." + str(N).zfill(D))[: 2 + digits]
    assert text.decode() == want


def test_prefix_consistency_pi_1e8(pic, golden):
    x = _pi_bf(pic, 100_000_000)
    long = x.to_dec(100_000_000)
    short = x.to_dec(1_000_000)
    mid = x.to_dec(12_345_678)
    assert len(long) == 100_000_002
    assert long.startswith(mid) and mid.startswith(short)
    # the leading digits are pi's, whatever the working precision
    g = golden["dec"]["pi"]["1000000"]
    assert long[:80].decode() == g["head"]
