// 64-bit modular arithmetic for the NTT kernels (host + device).
//
// Primes are < 2^63.  Two multiplication forms are used:
//  * Montgomery (R = 2^64): mont_mul(a, b) = a*b*R^-1 mod p, built on
//    mul.lo.u64 / mul.hi.u64.  Twiddles stored as w*R make mont_mul(x, wR) =
//    x*w, so data never has to enter or leave Montgomery form.
//  * Shoup (precomputed quotient, D. Harvey 2014): for a fixed twiddle w with
//    w' = floor(w * 2^64 / p), shoup_mul(x, w, w') = x*w mod p using one
//    mul.hi.u64 and two mul.lo.u64.
//
// The reference does the same products with a 128-bit product and a hardware
// 128/64 divide (_umul128 + _udiv128, NTT.cpp:85-90 and :277-282); a divide
// has no GPU equivalent, hence these forms.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define PIC_HD __host__ __device__ __forceinline__
#else
#define PIC_HD inline
#endif

namespace pic {

PIC_HD uint64_t mulhi64(uint64_t a, uint64_t b)
{
#if defined(__CUDA_ARCH__)
    return __umul64hi(a, b);
#else
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

// Modulus description shared by all kernels for one prime.
struct Mod64 {
    uint64_t p;         // prime, < 2^63
    uint64_t pinv_neg;  // -p^-1 mod 2^64
    uint64_t r2;        // R^2 mod p (R = 2^64)
};

PIC_HD uint64_t add_mod(uint64_t a, uint64_t b, uint64_t p)
{
    uint64_t s = a + b;  // a, b < p < 2^63: no wrap
    return s >= p ? s - p : s;
}

PIC_HD uint64_t sub_mod(uint64_t a, uint64_t b, uint64_t p)
{
    return a >= b ? a - b : a + (p - b);
}

// a * b * 2^-64 mod p for a*b < p * 2^64 (e.g. a < 2^64, b < p).
PIC_HD uint64_t mont_mul(uint64_t a, uint64_t b, uint64_t p, uint64_t pinv_neg)
{
    uint64_t lo = a * b;
    uint64_t hi = mulhi64(a, b);
    uint64_t m = lo * pinv_neg;
    // (a*b + m*p) / 2^64: the low halves sum to 0 mod 2^64, carrying 1 iff lo != 0.
    uint64_t r = hi + mulhi64(m, p) + (lo != 0);
    return r >= p ? r - p : r;
}

PIC_HD uint64_t mont_mul(uint64_t a, uint64_t b, const Mod64& m)
{
    return mont_mul(a, b, m.p, m.pinv_neg);
}

// mont_mul for p = c 2^32 + 1 (c < 2^30): -p^-1 mod 2^64 = c 2^32 - 1, so
// m = lo (c 2^32 - 1) needs one 32-bit multiply, and m p = m + (m c) 2^32
// gives hi(m p) from m c (64 x 32 bits) and one carry.  The result is below
// a b / 2^64 + p before its one correction: in [0, p) for a b < p 2^64, in
// [0, 2p) for operands below 4p of a prime below 2^61.
PIC_HD uint64_t mont_mul_c(uint64_t a, uint64_t b, uint64_t p, uint32_t c)
{
    const uint64_t lo = a * b;
    const uint64_t hi = mulhi64(a, b);
    const uint64_t m = ((uint64_t)((uint32_t)lo * c) << 32) - lo;
    const uint64_t x = (uint64_t)(uint32_t)m * c;               // m_lo c
    const uint64_t y = (uint64_t)(uint32_t)(m >> 32) * c + (x >> 32);  // (m c) >> 32
    const uint64_t s = (x << 32) + m;                            // low 64 bits of m c 2^32 + m
    const uint64_t mp_hi = y + (s < m);                          // hi(m p)
    const uint64_t r = hi + mp_hi + (lo != 0);
    return r >= p ? r - p : r;
}

// x * w mod p with ws = floor(w * 2^64 / p); x < 2^64, w < p.
PIC_HD uint64_t shoup_mul(uint64_t x, uint64_t w, uint64_t ws, uint64_t p)
{
    uint64_t q = mulhi64(x, ws);
    uint64_t r = x * w - q * p;  // true value in [0, 2p)
    return r >= p ? r - p : r;
}

// x * w mod p in [0, 2p) for any x < 2^64 (Shoup, ws = floor(w 2^64 / p)),
// for the product primes p = c 2^32 + 1: q = floor(x ws / 2^64) from all four
// 32 x 32 partial products, and q p mod 2^64 = q + ((q mod 2^32) c) 2^32.
PIC_HD uint64_t shoup_lazy32(uint64_t x, uint64_t w, uint64_t ws, uint32_t c)
{
#if defined(__CUDA_ARCH__)
    const uint32_t x0 = (uint32_t)x, x1 = (uint32_t)(x >> 32);
    const uint32_t s0 = (uint32_t)ws, s1 = (uint32_t)(ws >> 32);
    const uint32_t w0 = (uint32_t)w, w1 = (uint32_t)(w >> 32);
    uint32_t r0, r1;
    asm("{\n\t.reg .u32 u0, u1, u2, q0, q1;\n\t"
        "mul.hi.u32 u0, %2, %4;\n\t"
        "mad.lo.cc.u32 u0, %2, %5, u0;\n\t"
        "madc.hi.u32 u1, %2, %5, 0;\n\t"
        "mad.lo.cc.u32 u0, %3, %4, u0;\n\t"
        "madc.hi.cc.u32 u1, %3, %4, u1;\n\t"
        "addc.u32 u2, 0, 0;\n\t"
        "mad.lo.cc.u32 q0, %3, %5, u1;\n\t"
        "madc.hi.u32 q1, %3, %5, u2;\n\t"
        "mul.lo.u32 %0, %2, %6;\n\t"
        "mul.hi.u32 %1, %2, %6;\n\t"
        "mad.lo.u32 %1, %2, %7, %1;\n\t"
        "mad.lo.u32 %1, %3, %6, %1;\n\t"
        "mad.lo.u32 u1, q0, %8, q1;\n\t"
        "sub.cc.u32 %0, %0, q0;\n\t"
        "subc.u32 %1, %1, u1;\n\t"
        "}"
        : "=r"(r0), "=r"(r1)
        : "r"(x0), "r"(x1), "r"(s0), "r"(s1), "r"(w0), "r"(w1), "r"(c));
    return ((uint64_t)r1 << 32) | r0;
#else
    const uint64_t q = mulhi64(x, ws);
    return x * w - (q + ((uint64_t)((uint32_t)q * c) << 32));
#endif
}

// x * w mod p in [0, 4p) for any x < 2^64, p = c 2^32 + 1 below 2^61 (so
// 4p < 2^63).  The quotient keeps three of the four partial products of
// x ws: x1 s1 + hi(x1 s0) + hi(x0 s1) is floor(x ws / 2^64) minus at most 2
// (the dropped terms sum to less than 3 2^64), and the Shoup quotient itself
// is floor(x w / p) or one less, so x w - q p lies in [0, 4p).
#ifndef PIC_SHOUP_WIDE
#define PIC_SHOUP_WIDE 0
#endif
PIC_HD uint64_t shoup_approx32(uint64_t x, uint64_t w, uint64_t ws, uint32_t c)
{
#if defined(__CUDA_ARCH__) && PIC_SHOUP_WIDE
    // the same three partial products and corrections, with the 64-bit
    // accumulations as 32 x 32 -> 64 multiply-adds (mad.wide.u32)
    const uint32_t x0 = (uint32_t)x, x1 = (uint32_t)(x >> 32);
    const uint32_t s0 = (uint32_t)ws, s1 = (uint32_t)(ws >> 32);
    const uint32_t w0 = (uint32_t)w, w1 = (uint32_t)(w >> 32);
    uint32_t r0, r1;
    asm("{\n\t.reg .u32 t0, t1, q0, q1, u1;\n\t.reg .u64 t, q, xw;\n\t"
        "mul.hi.u32 t0, %2, %5;\n\t"
        "mad.hi.cc.u32 t0, %3, %4, t0;\n\t"
        "addc.u32 t1, 0, 0;\n\t"
        "mov.b64 t, {t0, t1};\n\t"
        "mad.wide.u32 q, %3, %5, t;\n\t"
        "mov.b64 {q0, q1}, q;\n\t"
        "mul.wide.u32 xw, %2, %6;\n\t"
        "mov.b64 {%0, %1}, xw;\n\t"
        "mad.lo.u32 %1, %2, %7, %1;\n\t"
        "mad.lo.u32 %1, %3, %6, %1;\n\t"
        "mad.lo.u32 u1, q0, %8, q1;\n\t"
        "sub.cc.u32 %0, %0, q0;\n\t"
        "subc.u32 %1, %1, u1;\n\t"
        "}"
        : "=r"(r0), "=r"(r1)
        : "r"(x0), "r"(x1), "r"(s0), "r"(s1), "r"(w0), "r"(w1), "r"(c));
    return ((uint64_t)r1 << 32) | r0;
#elif defined(__CUDA_ARCH__)
    const uint32_t x0 = (uint32_t)x, x1 = (uint32_t)(x >> 32);
    const uint32_t s0 = (uint32_t)ws, s1 = (uint32_t)(ws >> 32);
    const uint32_t w0 = (uint32_t)w, w1 = (uint32_t)(w >> 32);
    uint32_t r0, r1;
    asm("{\n\t.reg .u32 t0, t1, q0, q1, u1;\n\t"
        "mul.hi.u32 t0, %2, %5;\n\t"
        "mad.hi.cc.u32 t0, %3, %4, t0;\n\t"
        "addc.u32 t1, 0, 0;\n\t"
        "mad.lo.cc.u32 q0, %3, %5, t0;\n\t"
        "madc.hi.u32 q1, %3, %5, t1;\n\t"
        "mul.lo.u32 %0, %2, %6;\n\t"
        "mul.hi.u32 %1, %2, %6;\n\t"
        "mad.lo.u32 %1, %2, %7, %1;\n\t"
        "mad.lo.u32 %1, %3, %6, %1;\n\t"
        "mad.lo.u32 u1, q0, %8, q1;\n\t"
        "sub.cc.u32 %0, %0, q0;\n\t"
        "subc.u32 %1, %1, u1;\n\t"
        "}"
        : "=r"(r0), "=r"(r1)
        : "r"(x0), "r"(x1), "r"(s0), "r"(s1), "r"(w0), "r"(w1), "r"(c));
    return ((uint64_t)r1 << 32) | r0;
#else
    const uint64_t x0 = (uint32_t)x, x1 = x >> 32, s0 = (uint32_t)ws, s1 = ws >> 32;
    const uint64_t q = x1 * s1 + ((x1 * s0) >> 32) + ((x0 * s1) >> 32);
    return x * w - (q + ((uint64_t)((uint32_t)q * c) << 32));
#endif
}

// A 64-bit piece v < 2^64 < 9p (product primes above 2^64 / 9) brought into
// [0, 4p) by two conditional subtractions of 4p.
PIC_HD uint64_t piece_to_lazy(uint64_t v, uint64_t p4)
{
    v = v >= p4 ? v - p4 : v;
    return v >= p4 ? v - p4 : v;
}

// The same piece reduced to [0, p): [0, 4p) -> [0, 2p) -> [0, p).
PIC_HD uint64_t piece_to_strict(uint64_t v, uint64_t p)
{
    v = piece_to_lazy(v, 4 * p);
    v = v >= 2 * p ? v - 2 * p : v;
    return v >= p ? v - p : v;
}

// ---- host-only helpers (table construction) ------------------------------
inline uint64_t host_mulmod(uint64_t a, uint64_t b, uint64_t p)
{
    return (uint64_t)(((unsigned __int128)a * b) % p);
}

inline uint64_t host_powmod(uint64_t a, uint64_t e, uint64_t p)
{
    uint64_t r = 1 % p;
    a %= p;
    while (e) {
        if (e & 1) r = host_mulmod(r, a, p);
        a = host_mulmod(a, a, p);
        e >>= 1;
    }
    return r;
}

inline Mod64 make_mod(uint64_t p)
{
    Mod64 m;
    m.p = p;
    uint64_t inv = p;  // Newton: inv = p^-1 mod 2^64 (p odd)
    for (int i = 0; i < 6; i++) inv *= 2 - p * inv;
    m.pinv_neg = (uint64_t)0 - inv;
    unsigned __int128 r = (((unsigned __int128)1) << 64) % p;
    m.r2 = (uint64_t)((r * r) % p);
    return m;
}

inline uint64_t to_mont(uint64_t a, uint64_t p)  // a * 2^64 mod p
{
    return (uint64_t)((((unsigned __int128)(a % p)) << 64) % p);
}

inline uint64_t shoup_companion(uint64_t w, uint64_t p)  // floor(w * 2^64 / p)
{
    return (uint64_t)((((unsigned __int128)w) << 64) / p);
}

}  // namespace pic
