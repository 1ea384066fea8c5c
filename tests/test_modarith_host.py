"""Host build of the kernels' modular arithmetic header, checked against
128-bit arithmetic.

modarith.cuh is shared by host and device code; compiled here with g++ its
product forms (Montgomery, the special-form Montgomery for p = c 2^32 + 1,
Shoup) must agree with (a b) mod p computed through unsigned __int128 for the
three product primes.  The reference computes the same products with a
128-bit multiply and divide (NTT.cpp:85-90).
"""
from __future__ import annotations

import pathlib
import shutil
import subprocess

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
HEADER_DIR = ROOT / "piculator_b200" / "csrc"

PROGRAM = r"""
#include "modarith.cuh"
#include <cstdio>
using namespace pic;
typedef unsigned __int128 u128;
static uint64_t state = 0x243F6A8885A308D3ull;
static uint64_t next() {
    uint64_t z = (state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static uint64_t powmod(uint64_t b, uint64_t e, uint64_t p) {
    uint64_t r = 1;
    for (; e; e >>= 1, b = (uint64_t)((u128)b * b % p)) if (e & 1) r = (uint64_t)((u128)r * b % p);
    return r;
}
int main() {
    const uint64_t primes[3] = {4611685941117976577ull, 4611685692009873409ull, 4611685606110527489ull};
    long bad = 0;
    for (int k = 0; k < 3; ++k) {
        const uint64_t p = primes[k];
        const uint32_t c = (uint32_t)(p >> 32);
        if (((uint64_t)c << 32) + 1 != p) { std::printf("form %d\n", k); return 2; }
        uint64_t inv = 1;                            // p^-1 mod 2^64 by Newton
        for (int i = 0; i < 6; ++i) inv *= 2 - p * inv;
        const uint64_t pinv_neg = 0 - inv;
        const uint64_t rinv = powmod((uint64_t)(((u128)1 << 64) % p), p - 2, p);
        for (int i = 0; i < 200000; ++i) {
            uint64_t a = next(), b = next();
            // inputs as the kernels see them: fully reduced, lazy (< 2p) and extremes
            switch (i % 4) {
                case 0: a %= p; b %= p; break;
                case 1: a %= 2 * p; b %= p; break;
                case 2: a = (i & 8) ? p - 1 : 0; b %= p; break;
                default: a %= p; b = (i & 8) ? p - 1 : 1; break;
            }
            const uint64_t want = (uint64_t)((u128)((u128)a * b % p) * rinv % p);
            const uint64_t m1 = mont_mul(a, b, p, pinv_neg);
            const uint64_t m2 = mont_mul_c(a, b, p, c);
            const uint64_t w = b % p, ws = (uint64_t)(((u128)w << 64) / p);
            const uint64_t sh = shoup_mul(a % p, w, ws, p);
            const uint64_t want_sh = (uint64_t)((u128)(a % p) * w % p);
            if (m1 % p != want || m2 % p != want || m1 >= p || m2 >= p || sh != want_sh) ++bad;
        }
    }
    std::printf("%ld\n", bad);
    return bad != 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_product_forms_match_int128(tmp_path):
    src = tmp_path / "modarith_check.cpp"
    exe = tmp_path / "modarith_check"
    src.write_text(PROGRAM)
    subprocess.run(["g++", "-O2", "-std=c++17", f"-I{HEADER_DIR}", str(src), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip() == "0"
