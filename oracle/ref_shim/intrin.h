/* Linux stand-in for MSVC's <intrin.h>, force-included (-include) when the
 * reference sources are compiled in place by oracle/Makefile.  Test
 * infrastructure only: nothing in the product links this.
 *
 * Provides the few MSVC intrinsics the reference uses that GCC lacks
 * (_umul128 / _udiv128, used by NTT.cpp:85-90 and :277-282) and widens the
 * 16-byte _mm_malloc alignment of BigFloat.cpp:441-442 to 64 bytes, because
 * FFT.cpp:85 dereferences those buffers as __m256d (GCC emits aligned
 * 32-byte moves there; MSVC emits unaligned ones). */
#pragma once
#include <x86intrin.h>
#include <immintrin.h>
#include <sstream>
#include <atomic>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <cstdint>

static inline uint64_t _umul128(uint64_t a, uint64_t b, uint64_t* hi)
{
    unsigned __int128 r = (unsigned __int128)a * b;
    *hi = (uint64_t)(r >> 64);
    return (uint64_t)r;
}

/* MSVC's _udiv128 is the single x86-64 instruction DIV r/m64 (RDX:RAX / d),
 * which faults when the quotient does not fit in 64 bits.  The same
 * instruction here, rather than an unsigned __int128 division (a libgcc call
 * several times slower), so the reference's modmul (NTT.cpp:85-90, 277-282)
 * runs at the speed its author measured.  Every call site passes hi < d. */
static inline uint64_t _udiv128(uint64_t hi, uint64_t lo, uint64_t d, uint64_t* rem)
{
    uint64_t q, r;
    __asm__("divq %4" : "=a"(q), "=d"(r) : "a"(lo), "d"(hi), "rm"(d) : "cc");
    *rem = r;
    return q;
}

#define _mm_malloc(size, align) _mm_malloc((size), 64)
