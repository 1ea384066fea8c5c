"""Host build of the kernels' modular arithmetic header, checked against
128-bit arithmetic.

modarith.cuh is shared by host and device code; compiled here with g++ (the
host branches restate the device PTX quotient by quotient) its product forms
(Montgomery, the special-form Montgomery for p = c 2^32 + 1, exact and
three-partial-product Shoup, piece reduction) must agree with (a b) mod p
computed through unsigned __int128 for the three product primes, within the
lazy ranges the NTT kernels rely on.  The reference computes the same
products with a 128-bit multiply and divide (NTT.cpp:85-90).
"""
from __future__ import annotations

import pathlib
import re
import shutil
import subprocess

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
HEADER_DIR = ROOT / "piculator_b200" / "csrc"


def _product_primes() -> str:
    """The kProductPrimes initialiser, read from the engine's source."""
    src = (HEADER_DIR / "ntt.cu").read_text()
    m = re.search(r"kProductPrimes\[3\] = \{([^}]*)\}", src)
    assert m, "kProductPrimes not found"
    return m.group(1)


PRIMES = _product_primes()

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
    const uint64_t primes[3] = {PRIMES};
    long bad = 0;
    for (int k = 0; k < 3; ++k) {
        const uint64_t p = primes[k];
        const uint32_t c = (uint32_t)(p >> 32);
        if (((uint64_t)c << 32) + 1 != p || p >= (1ull << 61) || (u128)9 * p <= ((u128)1 << 64)) {
            std::printf("form %d\n", k);
            return 2;
        }
        uint64_t inv = 1;                            // p^-1 mod 2^64 by Newton
        for (int i = 0; i < 6; ++i) inv *= 2 - p * inv;
        const uint64_t pinv_neg = 0 - inv;
        const uint64_t rinv = powmod((uint64_t)(((u128)1 << 64) % p), p - 2, p);
        for (int i = 0; i < 200000; ++i) {
            uint64_t a = next(), b = next();
            // Montgomery operands as the kernels see them: reduced, lazy
            // forward outputs (< 4p) and extremes
            switch (i % 4) {
                case 0: a %= p; b %= p; break;
                case 1: a %= 4 * p; b %= 4 * p; break;
                case 2: a = (i & 8) ? 4 * p - 1 : 0; b %= 4 * p; break;
                default: a %= 4 * p; b = (i & 8) ? 4 * p - 1 : 1; break;
            }
            const uint64_t want = (uint64_t)((u128)((u128)a * b % p) * rinv % p);
            const uint64_t m2 = mont_mul_c(a, b, p, c);
            if (m2 % p != want || m2 >= 2 * p) ++bad;
            if (i % 4 == 0) {
                const uint64_t m1 = mont_mul(a, b, p, pinv_neg);
                if (m1 != want) ++bad;
            }
            // Shoup forms: any 64-bit x (lazy butterfly inputs reach 8p)
            const uint64_t x = (i % 3 == 0) ? next() : ((i % 3 == 1) ? next() % (8 * p) : ~0ull - (uint64_t)(i & 7));
            const uint64_t w = next() % p, ws = (uint64_t)(((u128)w << 64) / p);
            const uint64_t xw = (uint64_t)((u128)x * w % p);
            const uint64_t s1 = shoup_lazy32(x, w, ws, c), s2 = shoup_approx32(x, w, ws, c);
            if (s1 % p != xw || s1 >= 2 * p || s2 % p != xw || s2 >= 4 * p) ++bad;
            if (shoup_mul(x % p, w, ws, p) != xw) ++bad;
            const uint64_t v = next();
            const uint64_t lz = piece_to_lazy(v, 4 * p), st = piece_to_strict(v, p);
            if (lz % p != v % p || lz >= 4 * p || st != v % p) ++bad;
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
    src.write_text(PROGRAM.replace("PRIMES", PRIMES))
    subprocess.run(["g++", "-O2", "-std=c++17", f"-I{HEADER_DIR}", str(src), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.strip() == "0"
