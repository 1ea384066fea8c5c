// Modular arithmetic in FP64 for primes p < 2^47 (the FP64 product form).
//
// A residue is a double holding an integer, kept as a signed representative
// (|x| a small multiple of p, always below 2^51).  Every operation is exact:
//
//  * y w mod p for a fixed w with companion wp = fl(w / p) (Shoup's idea with
//    the quotient from the FP64 product): q = rint(y wp) from one fused
//    multiply-add with the rounding constant C = 1.5 2^52 (exact for
//    |y wp| < 2^51), h = fl(y w), l = y w - h exactly (fma), and
//    r = (h - q p) + l.  With |y| < 2^51 the quotient is within 0.75 of
//    y w / p, so |r| <= 0.75 p, and h - q p is an integer below 2^50 in
//    magnitude, hence exact; r + l is exact for the same reason.
//  * the same with the companion formed in place, wp = fl(w fl(1 / p))
//    (dmul_w, what the transforms use: their tables hold w alone): the
//    quotient is within 1 of y w / p, |r| <= p.
//  * a b mod p for two residues: the same with q = rint(h / p) from
//    fl(1 / p); |r| <= 0.75 p whenever |a b| < 2^51 p.
//  * reduction s mod p: s - rint(s / p) p, |r| <= p / 2 + 1 (for |s| < 2^56).
//
// The intrinsics (__fma_rn, __dmul_rn, __dadd_rn) keep the compiler from
// contracting or reassociating these steps.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pic {

constexpr double kDblRound = 6755399441055744.0;  // 1.5 * 2^52

__device__ __forceinline__ double dbits(uint64_t v) { return __longlong_as_double((long long)v); }
__device__ __forceinline__ uint64_t dstore(double d) { return (uint64_t)__double_as_longlong(d); }

// y * w mod p, |result| <= 0.75 p, for |y| < 2^51, 0 <= w < p, wp = fl(w / p).
__device__ __forceinline__ double dmul_tw(double y, double w, double wp, double p)
{
    const double q = __dadd_rn(__fma_rn(y, wp, kDblRound), -kDblRound);
    const double h = __dmul_rn(y, w);
    const double l = __fma_rn(y, w, -h);
    return __dadd_rn(__fma_rn(-q, p, h), l);
}

// y * w mod p with the companion formed here, wp = fl(w fl(1 / p)) (relative
// error below 2^-52, so the quotient is within 1 of y w / p): |result| <= p,
// for |y| < 2^51, 0 <= w < p.  The FP64 form's twiddle tables hold w alone.
__device__ __forceinline__ double dmul_w(double y, double w, double p, double pinv)
{
    return dmul_tw(y, w, __dmul_rn(w, pinv), p);
}

// a * b mod p, |result| <= 0.75 p, for |a b| < 2^51 p (|a|, |b| < 2^51).
__device__ __forceinline__ double dmul_mod(double a, double b, double p, double pinv)
{
    const double h = __dmul_rn(a, b);
    const double l = __fma_rn(a, b, -h);
    const double q = __dadd_rn(__fma_rn(h, pinv, kDblRound), -kDblRound);
    return __dadd_rn(__fma_rn(-q, p, h), l);
}

// s mod p, |result| <= p / 2 + 1, for any integer-valued |s| < 2^56.
__device__ __forceinline__ double dreduce(double s, double p, double pinv)
{
    const double q = __dadd_rn(__fma_rn(s, pinv, kDblRound), -kDblRound);
    return __fma_rn(-q, p, s);
}

// The representative in [0, p) of a residue with |x| < p.
__device__ __forceinline__ double dcanon(double x, double p) { return x < 0.0 ? __dadd_rn(x, p) : x; }

// A 56-bit piece v (< 2^56) as a residue, |result| <= p / 2 + 2^28:
// v = H 2^28 + L; H 2^28 and L are built exactly from their bits
// (2^80 + H 2^28 and 2^52 + L are doubles whose mantissas hold H and L).
__device__ __forceinline__ double dpiece56(uint64_t v, double p, double pinv)
{
    const uint32_t H = (uint32_t)(v >> 28), L = (uint32_t)v & 0x0fffffffu;
    const double h = __dadd_rn(__hiloint2double(0x44f00000, (int)H), -1208925819614629174706176.0);  // - 2^80
    const double l = __dadd_rn(__hiloint2double(0x43300000, (int)L), -4503599627370496.0);          // - 2^52
    return __dadd_rn(dreduce(h, p, pinv), l);
}

// Piece J of a word array x[0 .. n) in 56-bit pieces: bits 56 J .. 56 J + 55
// (zero above n words).  56 J mod 32 is 0, 8, 16 or 24, so a piece spans two
// words, or three when the shift passes 8.
__device__ __forceinline__ uint64_t src_piece56_raw(const uint32_t* __restrict__ x, uint32_t n, size_t J)
{
    const size_t bit = 56 * J;
    const size_t wi = bit >> 5;
    const int sh = (int)(bit & 31);
    const uint64_t w0 = wi < n ? __ldg(x + wi) : 0u;
    const uint64_t w1 = wi + 1 < n ? __ldg(x + wi + 1) : 0u;
    uint64_t v = (w0 | (w1 << 32)) >> sh;
    if (sh > 8 && wi + 2 < n) v |= (uint64_t)__ldg(x + wi + 2) << (64 - sh);
    return v & ((1ull << 56) - 1);
}

// A residue x with 0 <= x < 2^52 as an integer (the bits of x + 2^52).
__device__ __forceinline__ uint64_t dto_u64(double x)
{
    return (uint64_t)__double_as_longlong(__dadd_rn(x, 4503599627370496.0)) & ((1ull << 52) - 1);
}

}  // namespace pic
