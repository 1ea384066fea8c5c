"""The three-prime product forms' primes and the ranges their exactness rests
on, checked on the CPU from the constants in the CUDA sources.

* Integer form (kProductPrimes): primes c 2^32 + 1 between 2^64 / 9 and
  2^61; a convolution of 64-bit pieces whose shorter operand has at most
  2^30 pieces has coefficients below 2^158, and a merge's signed
  T1 +- T2 shifted by 2^159 per coefficient stays inside [0, p0 p1 p2).
* FP64 form (kDblPrimes): primes c 2^32 + 1 below 2^47 (16 p < 2^51, the
  FP64 quotient's range); 56-bit pieces with the shorter operand at most 2^28
  pieces give coefficients below 2^140 < p0 p1 p2, and the binary-splitting
  merges' signed sum shifted by 2^140 stays inside [0, p0 p1 p2) up to
  kDblMergeMaxPieces pieces (2^26).  2^27 pieces would not be safe in the
  worst case, which is why the limit is 2^26."""
from __future__ import annotations

import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "piculator_b200", "csrc")


def _src(name: str) -> str:
    with open(os.path.join(CSRC, name)) as f:
        return f.read()


def _primes(name: str) -> list[int]:
    m = re.search(name + r"\[3\]\s*=\s*\{([^}]*)\}", _src("ntt.cu"))
    assert m, name
    return [int(v.strip().rstrip("ull")) for v in m.group(1).split(",")]


def _is_prime(n: int) -> bool:
    """Deterministic Miller-Rabin for n < 3.3e24 (the first 13 prime bases)."""
    if n < 2:
        return False
    bases = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41)
    for b in bases:
        if n % b == 0:
            return n == b
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for b in bases:
        x = pow(b, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def _two_adicity(p: int) -> int:
    return ((p - 1) & -(p - 1)).bit_length() - 1


def test_integer_form_primes_and_ranges():
    P = _primes("kProductPrimes")
    assert len(set(P)) == 3
    for p in P:
        assert _is_prime(p) and (p - 1) % (1 << 32) == 0
        assert (1 << 64) // 9 < p < (1 << 61)
        assert _two_adicity(p) >= 32  # transforms up to 2^32 points
        assert 8 * p < (1 << 64)  # lazy inverse outputs in [0, 8p)
        assert 9 * p > (1 << 64) - 1  # a 64-bit piece is below 9p
    M = P[0] * P[1] * P[2]
    coef = (1 << 30) * ((1 << 64) - 1) ** 2
    assert coef < (1 << 158)
    # signed T1 +- T2 of two such products, shifted by 2^159
    assert (1 << 159) - 2 * coef > -(1 << 159) and (1 << 159) + 2 * coef < M


def test_fp64_form_primes_and_ranges():
    P = _primes("kDblPrimes")
    assert len(set(P)) == 3
    for p in P:
        assert _is_prime(p) and (p - 1) % (1 << 32) == 0
        assert p < (1 << 47) and 16 * p < (1 << 51)
    M = P[0] * P[1] * P[2]
    piece = (1 << 56) - 1
    assert (1 << 28) * piece ** 2 < (1 << 140) < M  # products: shorter operand <= 2^28 pieces
    m = re.search(r"kDblMergeMaxPieces\s*=\s*\(size_t\)1\s*<<\s*(\d+)", _src("bsr.cu"))
    assert m
    n = 1 << int(m.group(1))
    off = 1 << 140
    # the merges' signed sum of two products of at most n pieces, shifted by 2^140
    assert off - 2 * n * piece ** 2 >= 0 and off + 2 * n * piece ** 2 < M
    # twice the limit would leave the worst case outside [0, M)
    assert off + 2 * (2 * n) * piece ** 2 >= M


@pytest.mark.parametrize("name", ["kProductPrimes", "kDblPrimes"])
def test_primes_are_pairwise_coprime_with_crt_inverses(name):
    P = _primes(name)
    # Garner's constants exist: p0^-1 mod p1, (p0 p1)^-1 mod p2
    assert pow(P[0], -1, P[1]) * P[0] % P[1] == 1
    assert pow(P[0] * P[1], -1, P[2]) * (P[0] * P[1]) % P[2] == 1
