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

// x * w mod p with ws = floor(w * 2^64 / p); x < 2^64, w < p.
PIC_HD uint64_t shoup_mul(uint64_t x, uint64_t w, uint64_t ws, uint64_t p)
{
    uint64_t q = mulhi64(x, ws);
    uint64_t r = x * w - q * p;  // true value in [0, 2p)
    return r >= p ? r - p : r;
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
