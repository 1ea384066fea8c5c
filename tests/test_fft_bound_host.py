"""The FFT product form's piece width, from the library's host arithmetic
(pic_fft_piece_bits / pic_fft_error_bound, callable without a GPU) against
an independent restatement of the published bound: C. Percival, "Rapid
multiplication modulo the sum and difference of highly composite numbers",
Math. Comp. 72 (2003), Theorem 5.1 --
    err <= N X Y [(1 + e)^(3k) (1 + e sqrt 5)^(3k + 1) (1 + beta)^(3k) - 1]
with N = 2^k, X = Y = 2^b - 1, e = 2^-53 and beta = 2.5 e (each outer
twiddle the rounded product of two rounded table entries).  A piece width is
accepted while the bound stays below 1/4, so rounding the inverse transform
recovers every coefficient exactly."""
from __future__ import annotations

from fractions import Fraction

import pytest

import piculator_b200 as P


def _bound_exact(k: int, b: int) -> Fraction:
    """The bound in exact rational arithmetic, the powers expanded exactly
    (sqrt 5 replaced by a rational upper bound, so this errs high)."""
    e = Fraction(1, 2 ** 53)
    sqrt5_hi = Fraction(2236067977499790, 10 ** 15)  # > sqrt(5)
    beta = Fraction(5, 2) * e
    X = 2 ** b - 1
    growth = (1 + e) ** (3 * k) * (1 + e * sqrt5_hi) ** (3 * k + 1) * (1 + beta) ** (3 * k)
    return 2 ** k * X * X * (growth - 1)


def _bits_exact(k: int) -> int:
    for b in range(16, 7, -1):
        if _bound_exact(k, b) < Fraction(1, 4):
            return b
    return 0


@pytest.mark.parametrize("k", range(1, 31))
def test_piece_bits_match_the_published_bound(k):
    L = P.lib()
    assert L.pic_fft_piece_bits(k) == _bits_exact(k)


def test_piece_bits_table():
    """The widths quoted for the transform lengths of a pi run."""
    L = P.lib()
    got = {k: L.pic_fft_piece_bits(k) for k in (14, 17, 20, 23, 26, 27, 28)}
    assert got == {14: 14, 17: 12, 20: 11, 23: 9, 26: 8, 27: 0, 28: 0}


@pytest.mark.parametrize("k,b", [(10, 16), (20, 11), (20, 12), (26, 8), (27, 8)])
def test_error_bound_value(k, b):
    got = P.lib().pic_fft_error_bound(k, b)
    want = float(_bound_exact(k, b))
    assert got == pytest.approx(want, rel=1e-9)


def test_error_bound_rejects_bad_arguments():
    L = P.lib()
    assert L.pic_fft_error_bound(0, 8) == -1.0 and L.pic_fft_error_bound(20, 0) == -1.0
    assert L.pic_fft_piece_bits(0) == 0 and L.pic_fft_piece_bits(99) == 0
