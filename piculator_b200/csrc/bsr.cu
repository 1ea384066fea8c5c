// Batched Chudnovsky binary splitting (Pi_BSR, PI.h:64-136).
//
// The recursion tree splits [a, b) at m = (a + b) / 2, so every node at depth d
// has length floor(T / 2^d) or ceil(T / 2^d).  Below the depth where a merge
// could truncate (operands longer than p + 2 words or an add window wider than
// p + 2, BigFloat.cpp:337-366 and :196-200), every value is an exact integer
// and every merge is exact arithmetic: P = P0 Q1 + P1 R0, Q = Q0 Q1,
// R = R0 R1.  Those depths are evaluated level by level, all nodes of a depth
// in a few launches, with every value resident in HBM in fixed-capacity slots:
//   * bottom depth (node lengths 1 or 2): one thread per node, leaf formulas
//     (PI.h:67-88) and the two-leaf merge in registers;
//   * short children: one CTA per parent, schoolbook column sums and
//     carry-lookahead scans in shared memory;
//   * long children: batched three-prime NTT, each child transformed once and
//     reused by the two products that need it (the transform-domain reuse that
//     Transform.h was written for), CRT + carry per product, then a batched
//     signed add for P.
// The few top levels, where truncation happens, run through BigFloat exactly
// as the reference does.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "bigfloat.hpp"
#include "bsr.cuh"
#include "carry.cuh"
#include "common.cuh"
#include "fp64mod.cuh"
#include "mul.cuh"
#include "ntt.cuh"
#include "pi.cuh"

namespace pic {

// ---------------------------------------------------------------------------
// Per-depth storage.
struct Slots {
    size_t count = 0;
    uint32_t cap = 0;
    DevBuf<uint32_t> w;    // count x cap words
    DevBuf<uint32_t> len;  // count lengths (words, no leading zeros)
};

struct Level {
    size_t count = 0;
    Slots P, Q, R;
    DevBuf<uint8_t> sign;  // P's sign: 1 = positive or zero
    DevBuf<uint32_t> bnd;  // count + 1 boundaries a_0 < a_1 < ... < a_count = b
};

static void alloc_slots(Slots& s, size_t count, uint32_t cap, cudaStream_t st)
{
    s.count = count;
    s.cap = cap;
    s.w = DevBuf<uint32_t>(count * (size_t)cap, st);
    s.len = DevBuf<uint32_t>(count, st);
}

// Bits of Q(a,b) for any node of length <= n with b <= T: sum of log2 Q_j
// (PI.h:77-79), and likewise R (PI.h:81-84); |P| / Q <= sum |P_j| / Q_j
// <= n (0.09 + 3.6e-6 T) (R_j < Q_j makes the ratio subadditive).
static void slot_caps(double n, double T, uint32_t& cP, uint32_t& cQ, uint32_t& cR)
{
    const double lq = log2(10939058860032000.0) + 3.0 * log2(T + 1.0);
    const double lr = log2(72.0) + 3.0 * log2(T + 1.0);
    const double bq = n * lq, br = n * lr;
    const double bp = bq + log2(n * (0.0895 + 3.6e-6 * T) + 1.0) + 1.0;
    // margins: a product's words (na + nb, top word possibly zero) and P's
    // carry word fit in ceil(bound / 32) + 3 (+ 4 for P)
    cQ = (uint32_t)ceil(bq / 32.0) + 3;
    cR = (uint32_t)ceil(br / 32.0) + 3;
    cP = (uint32_t)ceil(bp / 32.0) + 4;
}

// ---------------------------------------------------------------------------
// Boundaries: child 2i = [a, m), child 2i+1 = [m, b), m = (a + b) / 2 (PI.h:90).
__global__ void split_bounds_kernel(const uint32_t* __restrict__ pb, size_t count, uint32_t* __restrict__ cb)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t a = pb[i], b = pb[i + 1];
        cb[2 * i] = a;
        cb[2 * i + 1] = (uint32_t)((a + b) / 2);
        if (i == count - 1) cb[2 * count] = b;
    }
}

// ---------------------------------------------------------------------------
// Small fixed-size multiword helpers (registers).
template <int N>
struct SW {
    uint32_t w[N];
    int n;  // used words, canonical (top nonzero) or 0
};

template <int N>
__device__ __forceinline__ void sw_set(SW<N>& x, uint64_t v)
{
#pragma unroll
    for (int i = 0; i < N; i++) x.w[i] = 0;
    x.w[0] = (uint32_t)v;
    if (N > 1) x.w[1] = (uint32_t)(v >> 32);
    x.n = (v >> 32) ? 2 : (v ? 1 : 0);
}

// x *= m (m a 32-bit word), the reference's mul(uint32_t) (BigFloat.cpp:156-183).
template <int N>
__device__ __forceinline__ void sw_mul_u32(SW<N>& x, uint32_t m)
{
    uint64_t carry = 0;
#pragma unroll
    for (int i = 0; i < N; i++) {
        if (i < x.n) {
            carry += (uint64_t)x.w[i] * m;
            x.w[i] = (uint32_t)carry;
            carry >>= 32;
        }
    }
    // the carry word lands at index x.n (static indexing keeps x in registers)
    const int n = x.n;
#pragma unroll
    for (int i = 0; i < N; i++)
        if (i == n && carry) x.w[i] = (uint32_t)carry;
    if (carry && n < N) x.n = n + 1;
}

// Canonical length: one past the highest nonzero word (static indexing keeps
// the words in registers).
template <int N>
__device__ __forceinline__ int sw_top(const SW<N>& x)
{
    int n = 0;
#pragma unroll
    for (int k = 0; k < N; k++)
        if (x.w[k] != 0) n = k + 1;
    return n;
}

// z = a * b over the full capacities (words past a.n / b.n are zero).
template <int NA, int NB, int NZ>
__device__ __forceinline__ void sw_mul(const SW<NA>& a, const SW<NB>& b, SW<NZ>& z)
{
    static_assert(NZ >= NA + NB, "product capacity");
#pragma unroll
    for (int i = 0; i < NZ; i++) z.w[i] = 0;
#pragma unroll
    for (int i = 0; i < NA; i++) {
        uint64_t carry = 0;
#pragma unroll
        for (int j = 0; j < NB; j++) {
            carry += (uint64_t)a.w[i] * b.w[j] + z.w[i + j];
            z.w[i + j] = (uint32_t)carry;
            carry >>= 32;
        }
        z.w[i + NB] = (uint32_t)carry;
    }
    z.n = sw_top(z);
}

// -1, 0, 1 as a <, ==, > b: the highest differing word decides.
template <int N>
__device__ __forceinline__ int sw_cmp(const SW<N>& a, const SW<N>& b)
{
    int c = 0;
#pragma unroll
    for (int i = 0; i < N; i++)
        if (a.w[i] != b.w[i]) c = a.w[i] < b.w[i] ? -1 : 1;
    return c;
}

// Signed sum: (sa, a) + (sb, b) -> (sz, z), the reference's add with
// sign dispatch (BigFloat.cpp:288-305) on exact integers.  N must leave room
// for the carry word.
template <int N>
__device__ __forceinline__ void sw_signed_add(bool sa, const SW<N>& a, bool sb, const SW<N>& b, bool& sz, SW<N>& z)
{
    if (sa == sb) {
        uint64_t c = 0;
#pragma unroll
        for (int i = 0; i < N; i++) {
            c += (uint64_t)a.w[i] + b.w[i];
            z.w[i] = (uint32_t)c;
            c >>= 32;
        }
        sz = sa;
    } else {
        const int c = sw_cmp(a, b);
        uint32_t br = 0;
#pragma unroll
        for (int i = 0; i < N; i++) {
            const uint32_t x = c >= 0 ? a.w[i] : b.w[i], y = c >= 0 ? b.w[i] : a.w[i];
            const uint64_t d = (uint64_t)x - y - br;
            z.w[i] = (uint32_t)d;
            br = (uint32_t)(d >> 63);
        }
        sz = c > 0 ? sa : (c < 0 ? sb : true);
    }
    z.n = sw_top(z);
    if (z.n == 0) sz = true;
}

// Leaf b (PI.h:67-88).
struct LeafV {
    SW<6> P;
    bool sP;
    SW<5> Q;
    SW<4> R;
};

__device__ __forceinline__ void leaf(uint32_t b, LeafV& v)
{
    sw_set(v.P, (uint64_t)b * 545140134ull + 13591409ull);
    sw_mul_u32(v.P, 2 * b - 1);
    sw_mul_u32(v.P, 6 * b - 5);
    sw_mul_u32(v.P, 6 * b - 1);
    v.sP = (b % 2) == 0;
    sw_set(v.Q, b);
    sw_mul_u32(v.Q, b);
    sw_mul_u32(v.Q, b);
    sw_mul_u32(v.Q, 26726400u);
    sw_mul_u32(v.Q, 409297880u);
    sw_set(v.R, 2 * b - 1);
    sw_mul_u32(v.R, 6 * b - 5);
    sw_mul_u32(v.R, 6 * b - 1);
}

template <int N>
__device__ __forceinline__ void store_sw(const SW<N>& x, uint32_t* slot, uint32_t cap, uint32_t* len)
{
#pragma unroll
    for (int i = 0; i < N; i++)
        if (i < (int)cap) slot[i] = x.w[i];
    *len = (uint32_t)x.n;
}

// Bottom depth: nodes of length 1 (a leaf) or 2 (two leaves merged).
__global__ void bottom_kernel(const uint32_t* __restrict__ bnd, size_t count,
                              uint32_t* Pw, uint32_t* Plen, uint8_t* Psign, uint32_t cP, uint32_t* Qw,
                              uint32_t* Qlen, uint32_t cQ, uint32_t* Rw, uint32_t* Rlen, uint32_t cR)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t a = bnd[i], b = bnd[i + 1];
        if (b - a == 1) {
            LeafV v;
            leaf(b, v);
            store_sw(v.P, Pw + i * cP, cP, Plen + i);
            Psign[i] = v.sP ? 1 : 0;
            store_sw(v.Q, Qw + i * cQ, cQ, Qlen + i);
            store_sw(v.R, Rw + i * cR, cR, Rlen + i);
        } else {
            LeafV l, r;
            leaf(a + 1, l);
            leaf(a + 2, r);
            SW<12> t1, t2, P;
            sw_mul(l.P, r.Q, t1);  // P0 Q1
            sw_mul(r.P, l.R, t2);  // P1 R0
            bool sP;
            sw_signed_add(l.sP, t1, r.sP, t2, sP, P);
            SW<10> Q;
            SW<8> R;
            sw_mul(l.Q, r.Q, Q);
            sw_mul(l.R, r.R, R);
            store_sw(P, Pw + i * cP, cP, Plen + i);
            Psign[i] = sP ? 1 : 0;
            store_sw(Q, Qw + i * cQ, cQ, Qlen + i);
            store_sw(R, Rw + i * cR, cR, Rlen + i);
        }
    }
}

// ---------------------------------------------------------------------------
// CTA-per-parent schoolbook merge.
//
// Shared-memory helpers; every thread of the block must call them.

// (s2:s1:s0) += a * b: one multiply-add into a 96-bit column sum.
__device__ __forceinline__ void mac96(uint32_t& s0, uint32_t& s1, uint32_t& s2, uint32_t a, uint32_t b)
{
    asm("mad.lo.cc.u32 %0, %3, %4, %0;\n\t"
        "madc.hi.cc.u32 %1, %3, %4, %1;\n\t"
        "addc.u32 %2, %2, 0;"
        : "+r"(s0), "+r"(s1), "+r"(s2)
        : "r"(a), "r"(b));
}

// Column sums col[3c..3c+2] = sum_i a_i b_(c-i) (96 bits) for the four
// columns c0 .. c0 + 3: a[i] is loaded once for all four, b slides through a
// four-word register window.
__device__ __forceinline__ void colsum4(const uint32_t* a, int na, const uint32_t* b, int nb, int c0, uint32_t zw,
                                        uint32_t* col)
{
    uint32_t s0[4] = {0, 0, 0, 0}, s1[4] = {0, 0, 0, 0}, s2[4] = {0, 0, 0, 0};
    const int ilo = max(0, c0 - nb + 1), ihi = min(c0 + 3, na - 1);
    uint32_t W[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
        const int j = c0 + u - ilo;
        W[u] = (j >= 0 && j < nb) ? b[j] : 0u;
    }
    for (int i = ilo; i <= ihi; i++) {
        const uint32_t ai = a[i];
#pragma unroll
        for (int u = 0; u < 4; u++) mac96(s0[u], s1[u], s2[u], ai, W[u]);
        W[3] = W[2];
        W[2] = W[1];
        W[1] = W[0];
        const int j = c0 - i - 1;
        W[0] = j >= 0 ? b[j] : 0u;
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
        const uint32_t c = (uint32_t)c0 + u;
        if (c < zw) {
            col[3 * c] = s0[u];
            col[3 * c + 1] = s1[u];
            col[3 * c + 2] = s2[u];
        }
    }
}

// z[0..na+nb) = a * b; col must hold 3 (na + nb) words.  Returns the length
// without leading zeros (0 if either operand is empty).
__device__ uint32_t cta_mul(const uint32_t* a, uint32_t na, const uint32_t* b, uint32_t nb, uint32_t* z,
                            uint32_t* col)
{
    if (na == 0 || nb == 0) {
        __syncthreads();
        return 0;
    }
    const uint32_t zw = na + nb;
    for (uint32_t g = threadIdx.x; 4 * g < zw; g += blockDim.x) colsum4(a, (int)na, b, (int)nb, (int)(4 * g), zw, col);
    __syncthreads();
    // each thread owns a contiguous run of output words
    const uint32_t per = (zw + blockDim.x - 1) / blockDim.x;
    const uint32_t w0 = threadIdx.x * per, w1 = min(w0 + per, zw);
    auto digit = [&](uint32_t w, uint32_t& g) -> uint32_t {
        uint64_t sw = col[3 * w], sp = 0;
        if (w >= 1) {
            sw += col[3 * (w - 1) + 1];
            sp += col[3 * (w - 1)];
        }
        if (w >= 2) {
            sw += col[3 * (w - 2) + 2];
            sp += col[3 * (w - 2) + 1];
        }
        if (w >= 3) sp += col[3 * (w - 3) + 2];
        const uint64_t t = (sw & 0xffffffffu) + (sp >> 32);
        g = (uint32_t)(t >> 32);
        return (uint32_t)t;
    };
    uint32_t gp = kGPIdentity;
    for (uint32_t w = w0; w < w1; w++) {
        uint32_t g;
        const uint32_t d = digit(w, g);
        gp = gp_combine(gp, g | ((uint32_t)(d == 0xffffffffu) << 1));
    }
    uint32_t total;
    uint32_t cin = block_gp_scan(gp, &total) & 1u;
    for (uint32_t w = w0; w < w1; w++) {
        uint32_t g;
        const uint32_t d = digit(w, g);
        z[w] = d + cin;
        cin = g | ((uint32_t)(d == 0xffffffffu) & cin);
    }
    __syncthreads();
    return z[zw - 1] == 0 ? zw - 1 : zw;
}

// Highest index < n with x[i] != 0, plus one (0 if none).
__device__ uint32_t cta_top(const uint32_t* x, uint32_t n)
{
    unsigned long long mine = 0;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
        if (x[i] != 0) mine = i + 1;
    return (uint32_t)block_max_u64(mine);
}

// z[0..zn) += x[0..xn) (sub: -=), in place, words of x past zn ignored; the
// caller guarantees the exact result fits zn words and is nonnegative.
__device__ void cta_add_into(uint32_t* z, uint32_t zn, const uint32_t* x, uint32_t xn, bool sub)
{
    const uint32_t per = (zn + blockDim.x - 1) / blockDim.x;
    const uint32_t w0 = threadIdx.x * per, w1 = min(w0 + per, zn);
    auto X = [&](uint32_t i) -> uint32_t { return i < xn ? x[i] : 0u; };
    uint32_t gp = kGPIdentity;
    for (uint32_t i = w0; i < w1; i++) {
        const uint32_t a = z[i], b = X(i);
        uint32_t d, g, p;
        if (!sub) {
            const uint64_t t = (uint64_t)a + b;
            d = (uint32_t)t;
            g = (uint32_t)(t >> 32);
            p = d == 0xffffffffu;
        } else {
            d = a - b;
            g = a < b;
            p = d == 0u;
        }
        gp = gp_combine(gp, g | (p << 1));
    }
    uint32_t total;
    uint32_t cin = block_gp_scan(gp, &total) & 1u;
    for (uint32_t i = w0; i < w1; i++) {
        const uint32_t a = z[i], b = X(i);
        if (!sub) {
            const uint64_t t = (uint64_t)a + b;
            const uint32_t d = (uint32_t)t;
            z[i] = d + cin;
            cin = (uint32_t)(t >> 32) | ((uint32_t)(d == 0xffffffffu) & cin);
        } else {
            const uint32_t d = a - b;
            z[i] = d - cin;
            cin = (uint32_t)(a < b) | ((uint32_t)(d == 0u) & cin);
        }
    }
    __syncthreads();
}

// z[0..na+nb) = a * b with one Karatsuba level when both operands are long
// enough: with h = min(na, nb) / 2, a = a1 B^h + a0, b = b1 B^h + b0,
//   z0 = a0 b0 and z2 = a1 b1 straight into z (disjoint halves),
//   m = (a0 + a1)(b0 + b1) - z0 - z2 = a0 b1 + a1 b0 (>= 0),
//   z += m B^h;
// three schoolbook products of about half the length instead of one: 3/4
// of the multiply-adds.  ws holds 3 (na + nb) + 8 words.  The words are those
// of the schoolbook product.
__device__ uint32_t cta_mul_k(const uint32_t* a, uint32_t na, const uint32_t* b, uint32_t nb, uint32_t* z,
                              uint32_t* col, uint32_t* ws, uint32_t kara_min)
{
    const uint32_t mn = min(na, nb);
    if (kara_min == 0 || mn < kara_min) return cta_mul(a, na, b, nb, z, col);
    const uint32_t zw = na + nb, h = mn / 2;
    const uint32_t la = na - h + 1, lb = nb - h + 1;  // sum lengths (carry word included)
    uint32_t* sa = ws;
    uint32_t* sb = sa + la;
    uint32_t* m = sb + lb;  // la + lb words
    // sa = a0 + a1, sb = b0 + b1 (na - h >= h words in a1, b1)
    for (uint32_t i = threadIdx.x; i < la; i += blockDim.x) sa[i] = i + h < na ? a[i + h] : 0u;
    for (uint32_t i = threadIdx.x; i < lb; i += blockDim.x) sb[i] = i + h < nb ? b[i + h] : 0u;
    __syncthreads();
    cta_add_into(sa, la, a, h, false);
    cta_add_into(sb, lb, b, h, false);
    // z0, z2 into z; m = sa sb
    cta_mul(a, h, b, h, z, col);
    cta_mul(a + h, na - h, b + h, nb - h, z + 2 * h, col);
    cta_mul(sa, la, sb, lb, m, col);
    cta_add_into(m, la + lb, z, 2 * h, true);
    cta_add_into(m, la + lb, z + 2 * h, zw - 2 * h, true);
    cta_add_into(z + h, zw - h, m, la + lb, false);
    return z[zw - 1] == 0 ? zw - 1 : zw;
}

// Signed sum of magnitudes (sa, a[0..na)) + (sb, b[0..nb)) into z (capacity
// max(na, nb) + 1).  Returns the length; *sz the sign.  Exact arithmetic
// with the reference's sign dispatch (BigFloat.cpp:288-305).
__device__ uint32_t cta_signed_add(bool sa, const uint32_t* a, uint32_t na, bool sb, const uint32_t* b, uint32_t nb,
                                   uint32_t* z, bool* sz)
{
    __shared__ int s_cmp;
    const uint32_t n = max(na, nb);
    auto A = [&](uint32_t i) -> uint32_t { return i < na ? a[i] : 0u; };
    auto B = [&](uint32_t i) -> uint32_t { return i < nb ? b[i] : 0u; };
    bool sub = sa != sb;
    bool swap = false;
    if (sub) {
        // compare magnitudes: highest differing word decides
        unsigned long long mine = 0;
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
            if (A(i) != B(i)) mine = i + 1;
        const uint32_t h = (uint32_t)block_max_u64(mine);
        if (threadIdx.x == 0) s_cmp = h == 0 ? 0 : (A(h - 1) > B(h - 1) ? 1 : -1);
        __syncthreads();
        const int c = s_cmp;
        __syncthreads();
        if (c == 0) {
            *sz = true;
            return 0;
        }
        swap = c < 0;
    }
    const uint32_t per = (n + blockDim.x - 1) / blockDim.x;
    const uint32_t w0 = threadIdx.x * per, w1 = min(w0 + per, n);
    uint32_t gp = kGPIdentity;
    for (uint32_t i = w0; i < w1; i++) {
        const uint32_t x = swap ? B(i) : A(i), y = swap ? A(i) : B(i);
        uint32_t d, g, p;
        if (!sub) {
            const uint64_t s = (uint64_t)x + y;
            d = (uint32_t)s;
            g = (uint32_t)(s >> 32);
            p = d == 0xffffffffu;
        } else {
            d = x - y;
            g = x < y;
            p = d == 0u;
        }
        gp = gp_combine(gp, g | (p << 1));
    }
    uint32_t total;
    uint32_t cin = block_gp_scan(gp, &total) & 1u;
    for (uint32_t i = w0; i < w1; i++) {
        const uint32_t x = swap ? B(i) : A(i), y = swap ? A(i) : B(i);
        if (!sub) {
            const uint64_t s = (uint64_t)x + y;
            const uint32_t d = (uint32_t)s;
            z[i] = d + cin;
            cin = (uint32_t)(s >> 32) | ((uint32_t)(d == 0xffffffffu) & cin);
        } else {
            const uint32_t d = x - y;
            z[i] = d - cin;
            cin = (uint32_t)(x < y) | ((uint32_t)(d == 0u) & cin);
        }
    }
    __syncthreads();
    uint32_t len;
    if (!sub) {
        if (threadIdx.x == 0) z[n] = total & 1u;
        __syncthreads();
        len = z[n] ? n + 1 : n;
        *sz = sa;
    } else {
        len = cta_top(z, n);
        *sz = swap ? sb : sa;
        if (len == 0) *sz = true;
    }
    __syncthreads();
    return len;
}

struct MergeArgs {
    // children (depth d + 1)
    const uint32_t *cPw, *cQw, *cRw, *cPl, *cQl, *cRl;
    const uint8_t* cS;
    uint32_t ccP, ccQ, ccR;
    // parents (depth d)
    uint32_t *pPw, *pQw, *pRw, *pPl, *pQl, *pRl;
    uint8_t* pS;
    uint32_t pcP, pcQ, pcR;
    size_t count;  // parents
    uint32_t kara_min;  // Karatsuba level for products whose operands both have this many words (0: never)
};

__global__ void __launch_bounds__(256) merge_school_kernel(MergeArgs m)
{
    extern __shared__ uint32_t sm[];
    const size_t i = blockIdx.x;
    const size_t L = 2 * i, R = 2 * i + 1;
    const uint32_t nPL = m.cPl[L], nQL = m.cQl[L], nRL = m.cRl[L];
    const uint32_t nPR = m.cPl[R], nQR = m.cQl[R], nRR = m.cRl[R];
    const bool sL = m.cS[L] != 0, sR = m.cS[R] != 0;
    uint32_t* PL = sm;
    uint32_t* QL = PL + m.ccP;
    uint32_t* RL = QL + m.ccQ;
    uint32_t* PR = RL + m.ccR;
    uint32_t* QR = PR + m.ccP;
    uint32_t* RR = QR + m.ccQ;
    uint32_t* t1 = RR + m.ccR;         // ccP + ccQ
    uint32_t* t2 = t1 + m.ccP + m.ccQ; // ccP + ccR
    uint32_t* col = t2 + m.ccP + m.ccR;  // 3 (ccP + ccQ) (the largest product)
    uint32_t* ws = col + 3 * (m.ccP + m.ccQ);  // Karatsuba sums and middle product
    for (uint32_t k = threadIdx.x; k < nPL; k += blockDim.x) PL[k] = m.cPw[L * m.ccP + k];
    for (uint32_t k = threadIdx.x; k < nQL; k += blockDim.x) QL[k] = m.cQw[L * m.ccQ + k];
    for (uint32_t k = threadIdx.x; k < nRL; k += blockDim.x) RL[k] = m.cRw[L * m.ccR + k];
    for (uint32_t k = threadIdx.x; k < nPR; k += blockDim.x) PR[k] = m.cPw[R * m.ccP + k];
    for (uint32_t k = threadIdx.x; k < nQR; k += blockDim.x) QR[k] = m.cQw[R * m.ccQ + k];
    for (uint32_t k = threadIdx.x; k < nRR; k += blockDim.x) RR[k] = m.cRw[R * m.ccR + k];
    __syncthreads();
    // Q = QL QR, R = RL RR written straight to the parent slots via t1 staging
    uint32_t nQ = cta_mul_k(QL, nQL, QR, nQR, t1, col, ws, m.kara_min);
    for (uint32_t k = threadIdx.x; k < nQ; k += blockDim.x) m.pQw[i * m.pcQ + k] = t1[k];
    uint32_t nR = cta_mul_k(RL, nRL, RR, nRR, t1, col, ws, m.kara_min);
    for (uint32_t k = threadIdx.x; k < nR; k += blockDim.x) m.pRw[i * m.pcR + k] = t1[k];
    __syncthreads();
    // P = PL QR + PR RL (PI.h:110)
    const uint32_t n1 = cta_mul_k(PL, nPL, QR, nQR, t1, col, ws, m.kara_min);
    const uint32_t n2 = cta_mul_k(PR, nPR, RL, nRL, t2, col, ws, m.kara_min);
    bool sP;
    uint32_t* pz = col;  // reuse: max(n1, n2) + 1 <= 3 (ccP + ccQ)
    const uint32_t nP = cta_signed_add(sL, t1, n1, sR, t2, n2, pz, &sP);
    for (uint32_t k = threadIdx.x; k < nP; k += blockDim.x) m.pPw[i * m.pcP + k] = pz[k];
    if (threadIdx.x == 0) {
        m.pPl[i] = nP;
        m.pQl[i] = nQ;
        m.pRl[i] = nR;
        m.pS[i] = sP ? 1 : 0;
    }
}

// ---------------------------------------------------------------------------
// Thread-per-parent merge for the shortest nodes: every operand and product
// in registers (fixed capacities CP, CQ, CR >= the child slots), fully
// unrolled word loops, the same results as merge_school_kernel.

template <int N>
__device__ __forceinline__ void sw_load(SW<N>& x, const uint32_t* __restrict__ w, uint32_t cap,
                                        const uint32_t* __restrict__ len, size_t c)
{
    const int n = (int)len[c];
    const uint32_t* src = w + c * (size_t)cap;
#pragma unroll
    for (int k = 0; k < N; k++) x.w[k] = k < n ? src[k] : 0u;
    x.n = n;
}

template <int NA, int NB>
__device__ __forceinline__ void sw_widen(const SW<NA>& a, SW<NB>& b)
{
#pragma unroll
    for (int k = 0; k < NB; k++) b.w[k] = k < NA ? a.w[k] : 0u;
    b.n = a.n;
}

template <int CP, int CQ, int CR>
__global__ void __launch_bounds__(128) merge_thread_kernel(MergeArgs m)
{
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= m.count) return;
    const size_t L = 2 * i, R = 2 * i + 1;
    {
        SW<CQ> a, b;
        sw_load(a, m.cQw, m.ccQ, m.cQl, L);
        sw_load(b, m.cQw, m.ccQ, m.cQl, R);
        SW<2 * CQ> z;
        sw_mul(a, b, z);
        store_sw(z, m.pQw + i * m.pcQ, m.pcQ, m.pQl + i);
    }
    {
        SW<CR> a, b;
        sw_load(a, m.cRw, m.ccR, m.cRl, L);
        sw_load(b, m.cRw, m.ccR, m.cRl, R);
        SW<2 * CR> z;
        sw_mul(a, b, z);
        store_sw(z, m.pRw + i * m.pcR, m.pcR, m.pRl + i);
    }
    // P = PL QR + PR RL (PI.h:110)
    constexpr int NP = CP + CQ + 1;
    SW<NP> t1, t2;
    {
        SW<CP> a;
        SW<CQ> b;
        sw_load(a, m.cPw, m.ccP, m.cPl, L);
        sw_load(b, m.cQw, m.ccQ, m.cQl, R);
        SW<CP + CQ> z;
        sw_mul(a, b, z);
        sw_widen(z, t1);
    }
    {
        SW<CP> a;
        SW<CR> b;
        sw_load(a, m.cPw, m.ccP, m.cPl, R);
        sw_load(b, m.cRw, m.ccR, m.cRl, L);
        SW<CP + CR> z;
        sw_mul(a, b, z);
        sw_widen(z, t2);
    }
    bool sP;
    SW<NP> P;
    sw_signed_add(m.cS[L] != 0, t1, m.cS[R] != 0, t2, sP, P);
    store_sw(P, m.pPw + i * m.pcP, m.pcP, m.pPl + i);
    m.pS[i] = sP ? 1 : 0;
}

template <int CP, int CQ, int CR>
static bool launch_merge_thread(const MergeArgs& m, cudaStream_t s)
{
    if (m.ccP > (uint32_t)CP || m.ccQ > (uint32_t)CQ || m.ccR > (uint32_t)CR) return false;
    merge_thread_kernel<CP, CQ, CR><<<(unsigned)((m.count + 127) / 128), 128, 0, s>>>(m);
    return true;
}

// ---------------------------------------------------------------------------
// Warp-per-parent schoolbook merge for short nodes (every child slot <= 64
// words): the same arithmetic as merge_school_kernel with warp-wide scans and
// __syncwarp instead of block barriers, several parents per CTA, and the six
// child operands fetched with independent loads.

constexpr int kWarpMergeMax = 64;  // largest child slot (words)
constexpr int kWarpMergeWarps = 8;

// Exclusive warp scan of one (g, p) per lane, lanes in position order.
__device__ __forceinline__ uint32_t warp_gp_scan(uint32_t gp, uint32_t* total)
{
    const int lane = threadIdx.x & 31;
    uint32_t v = gp;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, v, off);
        if (lane >= off) v = gp_combine(o, v);
    }
    uint32_t excl = __shfl_up_sync(0xffffffffu, v, 1);
    if (lane == 0) excl = kGPIdentity;
    *total = __shfl_sync(0xffffffffu, v, 31);
    return excl;
}

// z[0..na+nb) = a * b in the warp's shared region; col holds 3 (na + nb)
// words.  Returns the length without the leading zero word (0 if empty).
__device__ uint32_t warp_mul(const uint32_t* a, uint32_t na, const uint32_t* b, uint32_t nb, uint32_t* z,
                             uint32_t* col)
{
    const int lane = threadIdx.x & 31;
    if (na == 0 || nb == 0) return 0;
    const uint32_t zw = na + nb;
    for (uint32_t g = lane; 4 * g < zw; g += 32) colsum4(a, (int)na, b, (int)nb, (int)(4 * g), zw, col);
    __syncwarp();
    const uint32_t per = (zw + 31) / 32;
    const uint32_t w0 = lane * per, w1 = min(w0 + per, zw);
    auto digit = [&](uint32_t w, uint32_t& g) -> uint32_t {
        uint64_t sw = col[3 * w], sp = 0;
        if (w >= 1) {
            sw += col[3 * (w - 1) + 1];
            sp += col[3 * (w - 1)];
        }
        if (w >= 2) {
            sw += col[3 * (w - 2) + 2];
            sp += col[3 * (w - 2) + 1];
        }
        if (w >= 3) sp += col[3 * (w - 3) + 2];
        const uint64_t t = (sw & 0xffffffffu) + (sp >> 32);
        g = (uint32_t)(t >> 32);
        return (uint32_t)t;
    };
    uint32_t gp = kGPIdentity;
    for (uint32_t w = w0; w < w1; w++) {
        uint32_t g;
        const uint32_t d = digit(w, g);
        gp = gp_combine(gp, g | ((uint32_t)(d == 0xffffffffu) << 1));
    }
    uint32_t total;
    uint32_t cin = warp_gp_scan(gp, &total) & 1u;
    for (uint32_t w = w0; w < w1; w++) {
        uint32_t g;
        const uint32_t d = digit(w, g);
        z[w] = d + cin;
        cin = g | ((uint32_t)(d == 0xffffffffu) & cin);
    }
    __syncwarp();
    return z[zw - 1] == 0 ? zw - 1 : zw;
}

// Signed sum of magnitudes into z (capacity max(na, nb) + 1); the reference's
// sign dispatch (BigFloat.cpp:288-305) on exact operands.
__device__ uint32_t warp_signed_add(bool sa, const uint32_t* a, uint32_t na, bool sb, const uint32_t* b, uint32_t nb,
                                    uint32_t* z, bool* sz)
{
    const int lane = threadIdx.x & 31;
    const uint32_t n = max(na, nb);
    auto A = [&](uint32_t i) -> uint32_t { return i < na ? a[i] : 0u; };
    auto B = [&](uint32_t i) -> uint32_t { return i < nb ? b[i] : 0u; };
    const bool sub = sa != sb;
    bool swap = false;
    if (sub) {
        unsigned long long mine = 0;
        for (uint32_t i = lane; i < n; i += 32)
            if (A(i) != B(i)) mine = i + 1;
        const uint32_t h = (uint32_t)warp_max_u64(mine);
        if (h == 0) {
            *sz = true;
            return 0;
        }
        swap = A(h - 1) < B(h - 1);
    }
    const uint32_t per = (n + 31) / 32;
    const uint32_t w0 = lane * per, w1 = min(w0 + per, n);
    uint32_t gp = kGPIdentity;
    for (uint32_t i = w0; i < w1; i++) {
        const uint32_t x = swap ? B(i) : A(i), y = swap ? A(i) : B(i);
        uint32_t d, g, p;
        if (!sub) {
            const uint64_t s = (uint64_t)x + y;
            d = (uint32_t)s;
            g = (uint32_t)(s >> 32);
            p = d == 0xffffffffu;
        } else {
            d = x - y;
            g = x < y;
            p = d == 0u;
        }
        gp = gp_combine(gp, g | (p << 1));
    }
    uint32_t total;
    uint32_t cin = warp_gp_scan(gp, &total) & 1u;
    for (uint32_t i = w0; i < w1; i++) {
        const uint32_t x = swap ? B(i) : A(i), y = swap ? A(i) : B(i);
        if (!sub) {
            const uint64_t s = (uint64_t)x + y;
            const uint32_t d = (uint32_t)s;
            z[i] = d + cin;
            cin = (uint32_t)(s >> 32) | ((uint32_t)(d == 0xffffffffu) & cin);
        } else {
            const uint32_t d = x - y;
            z[i] = d - cin;
            cin = (uint32_t)(x < y) | ((uint32_t)(d == 0u) & cin);
        }
    }
    __syncwarp();
    if (!sub) {
        const uint32_t c = total & 1u;
        if (lane == 0) z[n] = c;
        __syncwarp();
        *sz = sa;
        return n + c;
    }
    unsigned long long mine = 0;
    for (uint32_t i = lane; i < n; i += 32)
        if (z[i] != 0) mine = i + 1;
    const uint32_t len = (uint32_t)warp_max_u64(mine);
    *sz = len == 0 ? true : (swap ? sb : sa);
    return len;
}

// Shared words per warp for child slots (cP, cQ, cR).
__host__ __device__ inline uint32_t warp_merge_words(uint32_t cP, uint32_t cQ, uint32_t cR)
{
    return 2 * (cP + cQ + cR) + (cP + cQ) + (cP + cR) + 3 * (cP + cQ);
}

__global__ void __launch_bounds__(32 * kWarpMergeWarps) merge_warp_kernel(MergeArgs m)
{
    extern __shared__ uint32_t sm[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const size_t i = (size_t)blockIdx.x * kWarpMergeWarps + wid;
    if (i >= m.count) return;  // whole warps leave together
    uint32_t* base = sm + (size_t)wid * warp_merge_words(m.ccP, m.ccQ, m.ccR);
    uint32_t* PL = base;
    uint32_t* QL = PL + m.ccP;
    uint32_t* RL = QL + m.ccQ;
    uint32_t* PR = RL + m.ccR;
    uint32_t* QR = PR + m.ccP;
    uint32_t* RR = QR + m.ccQ;
    uint32_t* t1 = RR + m.ccR;
    uint32_t* t2 = t1 + m.ccP + m.ccQ;
    uint32_t* col = t2 + m.ccP + m.ccR;
    const size_t L = 2 * i, R = 2 * i + 1;
    const uint32_t nPL = m.cPl[L], nQL = m.cQl[L], nRL = m.cRl[L];
    const uint32_t nPR = m.cPl[R], nQR = m.cQl[R], nRR = m.cRl[R];
    const bool sL = m.cS[L] != 0, sR = m.cS[R] != 0;
    // all six operands' loads issued before any is stored
    for (uint32_t k = lane; k < (uint32_t)kWarpMergeMax; k += 32) {
        const uint32_t pl = k < nPL ? m.cPw[L * m.ccP + k] : 0u;
        const uint32_t ql = k < nQL ? m.cQw[L * m.ccQ + k] : 0u;
        const uint32_t rl = k < nRL ? m.cRw[L * m.ccR + k] : 0u;
        const uint32_t pr = k < nPR ? m.cPw[R * m.ccP + k] : 0u;
        const uint32_t qr = k < nQR ? m.cQw[R * m.ccQ + k] : 0u;
        const uint32_t rr = k < nRR ? m.cRw[R * m.ccR + k] : 0u;
        if (k < nPL) PL[k] = pl;
        if (k < nQL) QL[k] = ql;
        if (k < nRL) RL[k] = rl;
        if (k < nPR) PR[k] = pr;
        if (k < nQR) QR[k] = qr;
        if (k < nRR) RR[k] = rr;
    }
    __syncwarp();
    const uint32_t nQ = warp_mul(QL, nQL, QR, nQR, t1, col);
    for (uint32_t k = lane; k < nQ; k += 32) m.pQw[i * m.pcQ + k] = t1[k];
    __syncwarp();
    const uint32_t nR = warp_mul(RL, nRL, RR, nRR, t1, col);
    for (uint32_t k = lane; k < nR; k += 32) m.pRw[i * m.pcR + k] = t1[k];
    __syncwarp();
    // P = PL QR + PR RL (PI.h:110)
    const uint32_t n1 = warp_mul(PL, nPL, QR, nQR, t1, col);
    const uint32_t n2 = warp_mul(PR, nPR, RL, nRL, t2, col);
    bool sP;
    uint32_t* pz = col;  // max(n1, n2) + 1 <= 3 (ccP + ccQ)
    const uint32_t nP = warp_signed_add(sL, t1, n1, sR, t2, n2, pz, &sP);
    for (uint32_t k = lane; k < nP; k += 32) m.pPw[i * m.pcP + k] = pz[k];
    if (lane == 0) {
        m.pPl[i] = nP;
        m.pQl[i] = nQ;
        m.pRl[i] = nR;
        m.pS[i] = sP ? 1 : 0;
    }
}

// ---------------------------------------------------------------------------
// Batched three-prime NTT merge.

// For every parent i and prime q (arrays laid out [q][child][stride], the
// transforms of length 2^k at the start of each item):
//   T1 = PL QR -> P[2i], T2 = PR RL -> P[2i+1], Q = QL QR -> Q[2i], R = RL RR -> R[2i]
// or, with the children's P signs `sgn` (parent i at sgn[2i], sgn[2i + 1]),
//   T1 +- T2 -> P[2i] (plus when the signs agree), nothing in P[2i+1].
__global__ void __launch_bounds__(256) merge_pointwise_kernel(uint64_t* __restrict__ P, uint64_t* __restrict__ Q,
                                                              uint64_t* __restrict__ R, uint32_t npar, int k,
                                                              size_t stride, uint32_t jbpr, Mod64 m0, Mod64 m1,
                                                              Mod64 m2, const uint8_t* __restrict__ sgn)
{
    // block -> (prime q, parent i, run of 512 points); two points per thread
    const uint32_t row = blockIdx.x / jbpr, jb = blockIdx.x - row * jbpr;
    const uint32_t q = row / npar, i = row - q * npar;
    const size_t j = ((size_t)jb * blockDim.x + threadIdx.x) * 2;
    if (j >= ((size_t)1 << k)) return;
    const Mod64& M = q == 0 ? m0 : (q == 1 ? m1 : m2);
    const uint32_t c = (uint32_t)(M.p >> 32);  // product primes c 2^32 + 1
    const size_t base = (size_t)q * 2 * npar;
    const size_t L = (base + 2 * (size_t)i) * stride + j, Rr = L + stride;
    const ulonglong2 pl = *reinterpret_cast<const ulonglong2*>(P + L), pr = *reinterpret_cast<const ulonglong2*>(P + Rr);
    const ulonglong2 ql = *reinterpret_cast<const ulonglong2*>(Q + L), qr = *reinterpret_cast<const ulonglong2*>(Q + Rr);
    const ulonglong2 rl = *reinterpret_cast<const ulonglong2*>(R + L), rr = *reinterpret_cast<const ulonglong2*>(R + Rr);
    if (sgn != nullptr) {
        // P[2i] = T1 + T2 if the children's P have one sign, T1 - T2 otherwise;
        // the products are in [0, 2p), so both forms stay in [0, 4p), inside
        // the inverse transform's input range
        const bool same = (sgn[2 * i] != 0) == (sgn[2 * i + 1] != 0);
        const uint64_t ax = mont_mul_c(pl.x, qr.x, M.p, c), ay = mont_mul_c(pl.y, qr.y, M.p, c);
        const uint64_t bx = mont_mul_c(pr.x, rl.x, M.p, c), by = mont_mul_c(pr.y, rl.y, M.p, c);
        const uint64_t p2 = 2 * M.p;
        *reinterpret_cast<ulonglong2*>(P + L) =
            same ? make_ulonglong2(ax + bx, ay + by) : make_ulonglong2(ax + p2 - bx, ay + p2 - by);
    } else {
        *reinterpret_cast<ulonglong2*>(P + L) = make_ulonglong2(mont_mul_c(pl.x, qr.x, M.p, c), mont_mul_c(pl.y, qr.y, M.p, c));
        *reinterpret_cast<ulonglong2*>(P + Rr) = make_ulonglong2(mont_mul_c(pr.x, rl.x, M.p, c), mont_mul_c(pr.y, rl.y, M.p, c));
    }
    *reinterpret_cast<ulonglong2*>(Q + L) = make_ulonglong2(mont_mul_c(ql.x, qr.x, M.p, c), mont_mul_c(ql.y, qr.y, M.p, c));
    *reinterpret_cast<ulonglong2*>(R + L) = make_ulonglong2(mont_mul_c(rl.x, rr.x, M.p, c), mont_mul_c(rl.y, rr.y, M.p, c));
}

// The same on FP64-form residues (signed doubles, fp64mod.cuh): forward
// outputs |x| <= p give products |y| <= 0.75 p (the quotient of a product
// below p^2 is off by far less than 1/4), and T1 +- T2 stays below 1.5 p,
// inside what the FP64 inverse accepts.
struct DblMod3 {
    double p[3], pinv[3];
};

__global__ void __launch_bounds__(256) merge_pointwise_d_kernel(uint64_t* __restrict__ P, uint64_t* __restrict__ Q,
                                                                uint64_t* __restrict__ R, uint32_t npar, int k,
                                                                size_t stride, uint32_t jbpr, DblMod3 M,
                                                                const uint8_t* __restrict__ sgn)
{
    const uint32_t row = blockIdx.x / jbpr, jb = blockIdx.x - row * jbpr;
    const uint32_t q = row / npar, i = row - q * npar;
    const size_t j = ((size_t)jb * blockDim.x + threadIdx.x) * 2;
    if (j >= ((size_t)1 << k)) return;
    const double p = q == 0 ? M.p[0] : (q == 1 ? M.p[1] : M.p[2]);
    const double pinv = q == 0 ? M.pinv[0] : (q == 1 ? M.pinv[1] : M.pinv[2]);
    const size_t base = (size_t)q * 2 * npar;
    const size_t L = (base + 2 * (size_t)i) * stride + j, Rr = L + stride;
    const double2 pl = *reinterpret_cast<const double2*>(P + L), pr = *reinterpret_cast<const double2*>(P + Rr);
    const double2 ql = *reinterpret_cast<const double2*>(Q + L), qr = *reinterpret_cast<const double2*>(Q + Rr);
    const double2 rl = *reinterpret_cast<const double2*>(R + L), rr = *reinterpret_cast<const double2*>(R + Rr);
    const double2 t1 = make_double2(dmul_mod(pl.x, qr.x, p, pinv), dmul_mod(pl.y, qr.y, p, pinv));
    const double2 t2 = make_double2(dmul_mod(pr.x, rl.x, p, pinv), dmul_mod(pr.y, rl.y, p, pinv));
    if (sgn != nullptr) {
        const bool same = (sgn[2 * i] != 0) == (sgn[2 * i + 1] != 0);
        *reinterpret_cast<double2*>(P + L) = same ? make_double2(__dadd_rn(t1.x, t2.x), __dadd_rn(t1.y, t2.y))
                                                  : make_double2(__dadd_rn(t1.x, -t2.x), __dadd_rn(t1.y, -t2.y));
    } else {
        *reinterpret_cast<double2*>(P + L) = t1;
        *reinterpret_cast<double2*>(P + Rr) = t2;
    }
    *reinterpret_cast<double2*>(Q + L) = make_double2(dmul_mod(ql.x, qr.x, p, pinv), dmul_mod(ql.y, qr.y, p, pinv));
    *reinterpret_cast<double2*>(R + L) = make_double2(dmul_mod(rl.x, rr.x, p, pinv), dmul_mod(rl.y, rr.y, p, pinv));
}

static void launch_merge_pointwise_d(uint64_t* P, uint64_t* Q, uint64_t* R, size_t npar, int k, size_t stride,
                                     const uint8_t* sgn, cudaStream_t s)
{
    PIC_REQUIRE(k >= 1 && stride % 2 == 0 && npar <= 0x7fffffffu / 3, PIC_ERR_INVALID, "pointwise merge shape");
    const uint32_t jbpr = (uint32_t)((((size_t)1 << k) + 511) / 512);
    const size_t blocks = 3 * npar * (size_t)jbpr;
    PIC_REQUIRE(blocks <= 0x7fffffffu, PIC_ERR_INVALID, "pointwise merge grid too large");
    DblMod3 M;
    for (int q = 0; q < 3; q++) {
        M.p[q] = (double)kDblPrimes[q];
        M.pinv[q] = 1.0 / M.p[q];
    }
    merge_pointwise_d_kernel<<<(unsigned)blocks, 256, 0, s>>>(P, Q, R, (uint32_t)npar, k, stride, jbpr, M, sgn);
}

// Launch over 3 primes x npar parents x 2^k points (stride even, 2^k >= 2).
static void launch_merge_pointwise(uint64_t* P, uint64_t* Q, uint64_t* R, size_t npar, int k, size_t stride,
                                   const Mod64& m0, const Mod64& m1, const Mod64& m2, const uint8_t* sgn,
                                   cudaStream_t s)
{
    PIC_REQUIRE(k >= 1 && stride % 2 == 0 && npar <= 0x7fffffffu / 3, PIC_ERR_INVALID, "pointwise merge shape");
    const uint32_t jbpr = (uint32_t)((((size_t)1 << k) + 511) / 512);
    const size_t blocks = 3 * npar * (size_t)jbpr;
    PIC_REQUIRE(blocks <= 0x7fffffffu, PIC_ERR_INVALID, "pointwise merge grid too large");
    merge_pointwise_kernel<<<(unsigned)blocks, 256, 0, s>>>(P, Q, R, (uint32_t)npar, k, stride, jbpr, m0, m1, m2,
                                                            sgn);
}


// Product lengths: z = a b with na, nb from the children; 0 if either is 0.
__global__ void product_len_kernel(const uint32_t* la, const uint32_t* lb, size_t c0, size_t npar, int a_off,
                                   int b_off, uint32_t* zl)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < npar; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t na = la[2 * (c0 + i) + a_off], nb = lb[2 * (c0 + i) + b_off];
        zl[i] = (na && nb) ? na + nb : 0;
    }
}

__global__ void fix_top_kernel(const uint32_t* w, uint32_t cap, uint32_t* len, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t l = len[i];
        if (l && w[i * (size_t)cap + l - 1] == 0) len[i] = l - 1;
    }
}

// CTA per parent: P = sL T1 + sR T2 over long operands, processed in chunks
// of blockDim * 8 words with the carry carried between chunks.
__global__ void __launch_bounds__(256) signed_add_kernel(const uint32_t* __restrict__ t1, const uint32_t* l1,
                                                         uint32_t c1, const uint32_t* __restrict__ t2,
                                                         const uint32_t* l2, uint32_t c2, const uint8_t* cS,
                                                         size_t c0, uint32_t* __restrict__ Pw, uint32_t* Pl,
                                                         uint8_t* Ps, uint32_t cP)
{
    const size_t i = blockIdx.x;
    const uint32_t na = l1[i], nb = l2[i];
    const bool sa = cS[2 * i] != 0, sb = cS[2 * i + 1] != 0;
    const uint32_t* a = t1 + i * (size_t)c1;
    const uint32_t* b = t2 + i * (size_t)c2;
    uint32_t* z = Pw + (c0 + i) * (size_t)cP;
    const uint32_t n = max(na, nb);
    const uint32_t nz = min(n, cP);  // words past the slot are zero in the result
    auto A = [&](uint32_t k) -> uint32_t { return k < na ? a[k] : 0u; };
    auto B = [&](uint32_t k) -> uint32_t { return k < nb ? b[k] : 0u; };
    const bool sub = sa != sb;
    bool swap = false;
    __shared__ uint32_t s_carry;
    if (sub) {
        // the highest differing word decides; it is almost always near the top,
        // so look at the top block of words first
        uint32_t h = 0;
        for (uint32_t top = n; top > 0 && h == 0;) {
            const uint32_t lo = top > blockDim.x ? top - blockDim.x : 0;
            const uint32_t k = lo + threadIdx.x;
            unsigned long long mine = (k < top && A(k) != B(k)) ? k + 1 : 0;
            h = (uint32_t)block_max_u64(mine);
            top = lo;
        }
        if (h == 0) {
            if (threadIdx.x == 0) {
                Pl[c0 + i] = 0;
                Ps[c0 + i] = 1;
            }
            return;
        }
        swap = A(h - 1) < B(h - 1);
    }
    constexpr int IPT = 8;
    const uint32_t chunk = blockDim.x * IPT;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < n; base += chunk) {
        const uint32_t cin_chunk = s_carry;
        const uint32_t w0 = base + threadIdx.x * IPT;
        uint32_t gp = kGPIdentity;
#pragma unroll
        for (int u = 0; u < IPT; u++) {
            const uint32_t k = w0 + u;
            uint32_t d = 0, g = 0, p = 1;
            if (k < n) {
                const uint32_t x = swap ? B(k) : A(k), y = swap ? A(k) : B(k);
                if (!sub) {
                    const uint64_t s = (uint64_t)x + y;
                    d = (uint32_t)s;
                    g = (uint32_t)(s >> 32);
                    p = d == 0xffffffffu;
                } else {
                    d = x - y;
                    g = x < y;
                    p = d == 0u;
                }
            }
            gp = gp_combine(gp, g | (p << 1));
        }
        uint32_t total;
        const uint32_t pre = block_gp_scan(gp, &total);
        uint32_t cin = (pre & 1u) | (((pre >> 1) & 1u) & cin_chunk);
#pragma unroll
        for (int u = 0; u < IPT; u++) {
            const uint32_t k = w0 + u;
            if (k >= nz) break;
            const uint32_t x = swap ? B(k) : A(k), y = swap ? A(k) : B(k);
            if (!sub) {
                const uint64_t s = (uint64_t)x + y;
                const uint32_t d = (uint32_t)s;
                z[k] = d + cin;
                cin = (uint32_t)(s >> 32) | ((uint32_t)(d == 0xffffffffu) & cin);
            } else {
                const uint32_t d = x - y;
                z[k] = d - cin;
                cin = (uint32_t)(x < y) | ((uint32_t)(d == 0u) & cin);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) s_carry = (total & 1u) | (((total >> 1) & 1u) & cin_chunk);
        __syncthreads();
    }
    if (!sub) {
        if (threadIdx.x == 0) {
            const uint32_t c = s_carry;
            if (c && n < cP) z[n] = 1;
            Pl[c0 + i] = n + (c ? 1 : 0);
            Ps[c0 + i] = sa ? 1 : 0;
        }
        return;
    }
    // strip leading zeros after a subtraction, scanning down from the top
    __syncthreads();
    uint32_t l = 0;
    for (uint32_t top = nz; top > 0 && l == 0;) {
        const uint32_t lo = top > blockDim.x ? top - blockDim.x : 0;
        const uint32_t k = lo + threadIdx.x;
        unsigned long long mine = (k < top && z[k] != 0) ? k + 1 : 0;
        l = (uint32_t)block_max_u64(mine);
        top = lo;
    }
    if (threadIdx.x == 0) {
        Pl[c0 + i] = l;
        Ps[c0 + i] = l == 0 ? 1 : ((swap ? sb : sa) ? 1 : 0);
    }
}

// ---- the same signed sum spread over many CTAs per parent -------------------
// For levels with few, long parents: one CTA per (parent, chunk of kWideWPC
// words), the chunks' carries (or borrows) joined by a segmented scan.
//   wide_cmp:    highest differing word of |T1|, |T2| per parent (atomicMax)
//   wide_k1:     chunk digits with in-chunk carries, chunk (G, P) aggregate
//   (carry_scan_segments: carry-in per chunk)
//   wide_ripple: +1 / -1 rippled into chunks with a carry-in
//   wide_final:  length (highest nonzero word, atomicMax), carry word, sign
constexpr int kWideIPT = 8;
constexpr uint32_t kWideWPC = 256 * kWideIPT;

struct WideAdd {
    const uint32_t *t1, *l1, *t2, *l2;
    uint32_t c1, c2;
    const uint8_t* cS;  // signs of the two addends of parent i at cS[2i], cS[2i + 1]
    size_t c0;          // first parent (level index)
    uint32_t *Pw, *Pl, cP;
    uint8_t* Ps;
    uint32_t* hd;    // per parent: highest differing word + 1
    uint32_t* agg;   // per (parent, chunk): (G, P), then carry-in
    uint32_t* aggc;  // per (parent, chunk): (G, P) kept for the final carry
    uint32_t cpp;    // chunks per parent
};

struct WideOp {
    bool sub, swap, zero;
};

__device__ __forceinline__ WideOp wide_op(const WideAdd& w, size_t i)
{
    WideOp o;
    const bool sa = w.cS[2 * i] != 0, sb = w.cS[2 * i + 1] != 0;
    o.sub = sa != sb;
    o.swap = false;
    o.zero = false;
    if (o.sub) {
        const uint32_t h = w.hd[i];
        if (h == 0) {
            o.zero = true;
        } else {
            const uint32_t na = w.l1[i], nb = w.l2[i];
            const uint32_t x = h - 1 < na ? w.t1[i * (size_t)w.c1 + h - 1] : 0u;
            const uint32_t y = h - 1 < nb ? w.t2[i * (size_t)w.c2 + h - 1] : 0u;
            o.swap = x < y;
        }
    }
    return o;
}

__global__ void __launch_bounds__(256) wide_cmp_kernel(WideAdd w)
{
    const size_t i = blockIdx.x / w.cpp, c = blockIdx.x % w.cpp;
    const uint32_t na = w.l1[i], nb = w.l2[i], n = max(na, nb);
    const uint32_t b0 = (uint32_t)c * kWideWPC;
    if (b0 >= n) return;
    const uint32_t* a = w.t1 + i * (size_t)w.c1;
    const uint32_t* b = w.t2 + i * (size_t)w.c2;
    unsigned long long mine = 0;
    for (uint32_t k = b0 + threadIdx.x; k < b0 + kWideWPC && k < n; k += blockDim.x) {
        const uint32_t x = k < na ? a[k] : 0u, y = k < nb ? b[k] : 0u;
        if (x != y) mine = k + 1;
    }
    mine = warp_max_u64(mine);
    if ((threadIdx.x & 31) == 0 && mine) atomicMax(w.hd + i, (uint32_t)mine);
}

__global__ void __launch_bounds__(256) wide_k1_kernel(WideAdd w)
{
    const size_t i = blockIdx.x / w.cpp, c = blockIdx.x % w.cpp;
    const uint32_t na = w.l1[i], nb = w.l2[i], n = max(na, nb);
    const WideOp o = wide_op(w, i);
    const uint32_t* a = w.t1 + i * (size_t)w.c1;
    const uint32_t* b = w.t2 + i * (size_t)w.c2;
    uint32_t* z = w.Pw + (w.c0 + i) * (size_t)w.cP;
    const uint32_t w0 = (uint32_t)c * kWideWPC + threadIdx.x * kWideIPT;
    auto X = [&](uint32_t k) -> uint32_t {
        const uint32_t u = k < na ? a[k] : 0u, v = k < nb ? b[k] : 0u;
        return o.swap ? v : u;
    };
    auto Y = [&](uint32_t k) -> uint32_t {
        const uint32_t u = k < na ? a[k] : 0u, v = k < nb ? b[k] : 0u;
        return o.swap ? u : v;
    };
    uint32_t gp = kGPIdentity;
    uint32_t xs[kWideIPT], ys[kWideIPT];
#pragma unroll
    for (int u = 0; u < kWideIPT; u++) {
        const uint32_t k = w0 + u;
        xs[u] = k < n ? X(k) : 0u;
        ys[u] = k < n ? Y(k) : 0u;
        uint32_t g = 0, p = 1;
        if (k < n) {
            if (!o.sub) {
                const uint64_t sum = (uint64_t)xs[u] + ys[u];
                g = (uint32_t)(sum >> 32);
                p = (uint32_t)sum == 0xffffffffu;
            } else {
                g = xs[u] < ys[u];
                p = xs[u] == ys[u];
            }
        }
        gp = gp_combine(gp, g | (p << 1));
    }
    uint32_t total;
    uint32_t cin = block_gp_scan(gp, &total) & 1u;
#pragma unroll
    for (int u = 0; u < kWideIPT; u++) {
        const uint32_t k = w0 + u;
        if (k >= n || k >= w.cP || o.zero) break;  // words past the slot are zero in the result
        if (!o.sub) {
            const uint64_t sum = (uint64_t)xs[u] + ys[u];
            const uint32_t d = (uint32_t)sum;
            z[k] = d + cin;
            cin = (uint32_t)(sum >> 32) | ((uint32_t)(d == 0xffffffffu) & cin);
        } else {
            const uint32_t d = xs[u] - ys[u];
            z[k] = d - cin;
            cin = (uint32_t)(xs[u] < ys[u]) | ((uint32_t)(d == 0u) & cin);
        }
    }
    if (threadIdx.x == 0) {
        w.agg[blockIdx.x] = total;
        w.aggc[blockIdx.x] = total;
    }
}

// Chunks with a carry-in: +1 (add) or -1 (subtract) rippled from the chunk's
// first word to the first word that absorbs it.
__global__ void __launch_bounds__(256) wide_ripple_kernel(WideAdd w)
{
    if (w.agg[blockIdx.x] == 0) return;
    const size_t i = blockIdx.x / w.cpp, c = blockIdx.x % w.cpp;
    const uint32_t n = max(w.l1[i], w.l2[i]);
    const WideOp o = wide_op(w, i);
    if (o.zero) return;
    uint32_t* z = w.Pw + (w.c0 + i) * (size_t)w.cP;
    const uint32_t b0 = (uint32_t)c * kWideWPC, e = min(min(b0 + kWideWPC, n), w.cP);
    if (b0 >= e) return;
    const uint32_t stop = o.sub ? 0u : 0xffffffffu;  // words that pass the carry on
    unsigned long long mine = ~0ull;
    for (uint32_t k = b0 + threadIdx.x; k < e; k += blockDim.x)
        if (z[k] != stop && k < mine) mine = k;
    const uint32_t f = (uint32_t)min((unsigned long long)e, block_min_u64(mine));
    for (uint32_t k = b0 + threadIdx.x; k < f; k += blockDim.x) z[k] = ~stop;
    if (threadIdx.x == 0 && f < e) z[f] += o.sub ? 0xffffffffu : 1u;
}

// Length, carry word and sign.  Parent lengths start at zero.
__global__ void __launch_bounds__(256) wide_final_kernel(WideAdd w)
{
    const size_t i = blockIdx.x / w.cpp, c = blockIdx.x % w.cpp;
    const uint32_t n = max(w.l1[i], w.l2[i]);
    const WideOp o = wide_op(w, i);
    const bool sa = w.cS[2 * i] != 0, sb = w.cS[2 * i + 1] != 0;
    uint32_t* z = w.Pw + (w.c0 + i) * (size_t)w.cP;
    if (!o.sub) {
        // the carry out of the last chunk: its (G, P) joined with its carry-in
        const uint32_t last = n ? (n - 1) / kWideWPC : 0;
        if (c == last && threadIdx.x == 0) {
            const uint32_t gp = w.aggc[blockIdx.x], cin = w.agg[blockIdx.x];
            const uint32_t carry = n ? ((gp & 1u) | ((gp >> 1) & cin)) : 0u;
            if (carry && n < w.cP) z[n] = 1;
            w.Pl[w.c0 + i] = n + carry;
            w.Ps[w.c0 + i] = sa ? 1 : 0;
        }
        return;
    }
    if (c == 0 && threadIdx.x == 0) w.Ps[w.c0 + i] = o.zero ? 1 : ((o.swap ? sb : sa) ? 1 : 0);
    if (o.zero) return;
    const uint32_t b0 = (uint32_t)c * kWideWPC, e = min(min(b0 + kWideWPC, n), w.cP);
    unsigned long long mine = 0;
    for (uint32_t k = b0 + threadIdx.x; k < e; k += blockDim.x)
        if (z[k] != 0) mine = k + 1;
    mine = warp_max_u64(mine);
    if ((threadIdx.x & 31) == 0 && mine) atomicMax(w.Pl + w.c0 + i, (uint32_t)mine);
}

static inline int ceil_log2_sz(size_t n)
{
    int k = 0;
    while (((size_t)1 << k) < n) k++;
    return k;
}

// The three primes' constants for the pointwise kernel.
static Mod64 prime_mod(int q) { return make_mod(kProductPrimes[q]); }

static bool g_wrap = true;
static uint32_t g_kara_min = 0;  // CTA schoolbook merges: Karatsuba level from this many words (0: off)
static int g_small_merge = 2;  // 0: CTA schoolbook, 1: + warp per parent, 2: + thread per parent
static bool g_top_batched = true;
static bool g_wide_add = true;

// Parameters of one level's batched NTT merge.  Every operand has at most
// smax pieces (ceil(cmax / 2) of 64 bits, or in the FP64 form
// ceil(32 cmax / 56) of 56 bits), every product at most L = 2 smax - 1
// coefficients.  Plain form: one transform of length 2^ceil_log2(L).  Wrapped
// form (when L sits just above a power of two): main length Nm = 2^(k-1) plus
// a tail product of length T >= 2W - 1 over the top W = L - Nm pieces.
struct MergeShape {
    int form = kFormInt;  // three-prime form of the level
    int k = 0;            // main transform bits
    size_t N = 0;         // main length
    size_t stride = 0;    // item stride of the main arrays (>= N + W)
    bool wrap = false;
    int kt = 0;           // tail transform bits
    size_t T = 0, W = 0, t0 = 0;
};

// The FP64 form serves a level while 2 smax (2^56)^2 + 2^140 < p0 p1 p2:
// smax <= 2^26 pieces (the signed combined P with its offset).
constexpr size_t kDblMergeMaxPieces = (size_t)1 << 26;

static MergeShape merge_shape(uint32_t cmax)
{
    MergeShape m;
    {
        const size_t si = ((size_t)cmax + 1) / 2, sd = pieces56(cmax);
        m.form = (sd <= kDblMergeMaxPieces && ntt_form_for(si, si, sd, sd, g_wrap) == kFormDbl) ? kFormDbl : kFormInt;
    }
    const size_t smax = m.form == kFormDbl ? pieces56(cmax) : ((size_t)cmax + 1) / 2;
    const size_t L = smax ? 2 * smax - 1 : 1;
    int k = ceil_log2_sz(L);
    if (k < 2) k = 2;
    PIC_REQUIRE(k <= 30, PIC_ERR_LENGTH, "binary-splitting node too long for the three-prime NTT");
    m.k = k;
    m.N = (size_t)1 << k;
    m.stride = m.N;
    const size_t Nm = m.N / 2;
    if (g_wrap && k >= 4 && smax <= Nm && L > Nm) {
        const size_t W = L - Nm;
        int kt = ceil_log2_sz(2 * W - 1);
        if (kt < 2) kt = 2;
        if (((size_t)1 << kt) <= Nm / 2) {
            m.wrap = true;
            m.k = k - 1;
            m.N = Nm;
            m.W = W;
            m.kt = kt;
            m.T = (size_t)1 << kt;
            m.t0 = Nm - smax + 1;
            m.stride = Nm + ((W + 15) & ~(size_t)15);
        }
    }
    return m;
}

// Destinations of the four products of a batch of parents (np of them):
// T1 = PL QR and T2 = PR RL at T1 + i c1 / T2 + i c2, Q = QL QR and R = RL RR
// at Q + i cQ / R + i cR, lengths (leading zero word dropped) in l1, l2, lQ,
// lR.  R == nullptr skips R.
struct ProductsOut {
    uint32_t* T1 = nullptr;
    uint32_t c1 = 0;
    uint32_t* l1 = nullptr;
    uint32_t* T2 = nullptr;
    uint32_t c2 = 0;
    uint32_t* l2 = nullptr;
    uint32_t* Q = nullptr;
    uint32_t cQ = 0;
    uint32_t* lQ = nullptr;
    uint32_t* R = nullptr;
    uint32_t cR = 0;
    uint32_t* lR = nullptr;
    // Combined mode (csign != null, the children's P signs, parent i at
    // csign[2i]): T1 receives V + K, V = T1 +- T2 (minus when the signs
    // differ), K = sum_(j < ncoef) 2^(159 + 64 j), with ncoef from
    // products_ncoef; c1 >= 2 ncoef + 6, l1 is set to 2 ncoef + 6; T2 unused.
    const uint8_t* csign = nullptr;
};

// Coefficients the batched products of a level convert (main transform plus
// wrapped top coefficients).
static size_t products_ncoef(const MergeShape& sh) { return sh.wrap ? sh.N + sh.W : sh.N; }

// Words of V + K in the combined form (every coefficient plus the offset:
// below 2^160 at bit 64 j, or below 2^141 at bit 56 j in the FP64 form), and
// of K alone.
static uint32_t combined_words(const MergeShape& sh, size_t ncoef)
{
    return sh.form == kFormDbl ? (uint32_t)((56 * ncoef + 86 + 31) / 32 + 1) : (uint32_t)(2 * ncoef + 6);
}
static uint32_t offset_words(const MergeShape& sh, size_t ncoef)
{
    return sh.form == kFormDbl ? (uint32_t)(((140 + 56 * (ncoef - 1)) >> 5) + 1) : (uint32_t)(2 * ncoef + 3);
}

__global__ void fill_u32_kernel(uint32_t* p, size_t n, uint32_t v)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}

// Bytes of transform storage per parent for a level's NTT merge.
static size_t ntt_bytes_per_parent(const MergeShape& sh) { return 3 * 2 * 3 * (sh.stride + sh.T) * sizeof(uint64_t); }

// The products of parents [p0, p0 + np) of the level above `ch`: each child
// operand is transformed once (six forward transforms per parent, four
// inverse), every product exact.
static void ntt_products(const Level& ch, size_t p0, size_t np, const MergeShape& sh, const ProductsOut& o,
                         cudaStream_t s, bool use_workspace = false)
{
    const uint32_t ccP = ch.P.cap, ccQ = ch.Q.cap, ccR = ch.R.cap;
    const uint32_t cmax = std::max(ccP, std::max(ccQ, ccR));
    const int k = sh.k;
    const size_t N = sh.N, ST = sh.stride, T = sh.T;
    const Mod64 m0 = prime_mod(0), m1 = prime_mod(1), m2 = prime_mod(2);
    const bool needR = o.R != nullptr;
    const bool dbl = sh.form == kFormDbl;
    // tail scale Nm / T in Montgomery form (mont_mul(x, c) = x Nm / T)
    uint64_t cT[3] = {0, 0, 0};
    if (sh.wrap && !dbl)
        for (int q = 0; q < 3; q++) cT[q] = to_mont((uint64_t)(N / T), kProductPrimes[q]);
    const size_t ncoef = products_ncoef(sh);
    {
        const size_t nc = 2 * np, c0 = 2 * p0;
        // six work arrays: from the persistent workspace when asked (the
        // top levels), else from the pool
        const size_t nmain = 3 * nc * ST, ntail = sh.wrap ? 3 * nc * T : 0;
        const size_t smain = (nmain + 31) & ~(size_t)31, stail = (ntail + 31) & ~(size_t)31;  // 256-byte steps
        WorkspaceLease ws(use_workspace ? 8 * (3 * smain + 3 * stail) : 0, s);
        DevBuf<uint64_t> owned[6];
        uint64_t* arr[6];
        for (int q = 0; q < 6; q++) {
            const size_t n = q < 3 ? nmain : ntail;
            if (ws.ptr) arr[q] = static_cast<uint64_t*>(ws.ptr) + (q < 3 ? q * smain : 3 * smain + (q - 3) * stail);
            else {
                owned[q] = DevBuf<uint64_t>(n, s);
                arr[q] = owned[q].get();
            }
        }
        uint64_t* const PB = arr[0];
        uint64_t* const QB = arr[1];
        uint64_t* const RB = arr[2];
        uint64_t* const PT = arr[3];
        uint64_t* const QT = arr[4];
        uint64_t* const RT = arr[5];
        NttBatch fb;
        fb.stride = ST;
        fb.count = (int)(3 * nc);
        fb.per_prime = (int)nc;
        for (int q = 0; q < 3; q++)
            fb.prime[q] = dbl ? dbl_prime_tables(kDblPrimes[q]).dev : prime_tables(kProductPrimes[q]).dev;
        NttBatch tb = fb;
        tb.stride = T;
        // the children's words are split into residues by each transform's
        // first pass (SplitSrc): main transforms from piece 0, tails from t0
        const Slots* arrays[3] = {&ch.P, &ch.Q, &ch.R};
        uint64_t* mains[3] = {PB, QB, RB};
        uint64_t* tails[3] = {PT, QT, RT};
        for (int a = 0; a < 3; a++) {
            SplitSrc src;
            src.words = arrays[a]->w.get();
            src.len = arrays[a]->len.get();
            src.cap = arrays[a]->cap;
            src.c0 = c0;
            src.first = 0;
            fb.data = mains[a];
            fb.src = src;
            ntt_forward_dif(fb, k, s);
            if (sh.wrap) {
                src.first = sh.t0;
                tb.data = tails[a];
                tb.src = src;
                ntt_forward_dif(tb, sh.kt, s);
            }
        }
        fb.src = SplitSrc{};
        tb.src = SplitSrc{};
        {
            ProfScope ps(KC_NTT_POINTWISE, 3.0 * 3 * np * (double)(N + T) * 80.0 / 8.0, s);
            if (dbl) {
                launch_merge_pointwise_d(PB, QB, RB, np, k, ST, o.csign, s);
                if (sh.wrap) launch_merge_pointwise_d(PT, QT, RT, np, sh.kt, T, o.csign, s);
            } else {
                launch_merge_pointwise(PB, QB, RB, np, k, ST, m0, m1, m2, o.csign, s);
                if (sh.wrap) launch_merge_pointwise(PT, QT, RT, np, sh.kt, T, m0, m1, m2, o.csign, s);
            }
            PIC_CHECK_LAUNCH();
            count_launch(sh.wrap ? 2 : 1);
        }
        // inverses: P holds T1, T2 for every parent (all items), or only the
        // combined item 2i; Q, R the even items
        const bool comb = o.csign != nullptr;
        {
            NttBatch eb = fb;
            eb.stride = 2 * ST;
            eb.count = (int)(3 * np);
            eb.per_prime = (int)np;
            if (comb) {
                eb.data = PB;
                ntt_inverse_dit(eb, k, s);
            } else {
                NttBatch ib = fb;
                ib.data = PB;
                ntt_inverse_dit(ib, k, s);
            }
            eb.data = QB;
            ntt_inverse_dit(eb, k, s);
            if (needR) {
                eb.data = RB;
                ntt_inverse_dit(eb, k, s);
            }
        }
        if (sh.wrap) {
            NttBatch eb = tb;
            eb.stride = 2 * T;
            eb.count = (int)(3 * np);
            eb.per_prime = (int)np;
            if (comb) {
                eb.data = PT;
                ntt_inverse_dit(eb, sh.kt, s);
            } else {
                NttBatch ib = tb;
                ib.data = PT;
                ntt_inverse_dit(ib, sh.kt, s);
            }
            eb.data = QT;
            ntt_inverse_dit(eb, sh.kt, s);
            if (needR) {
                eb.data = RT;
                ntt_inverse_dit(eb, sh.kt, s);
            }
            ProfScope ps(KC_NTT_POINTWISE, 3.0 * 4 * np * (double)sh.W * 24.0, s);
            const size_t W = sh.W;
            auto fix = [&](uint64_t* y, const uint64_t* tail, size_t nitems, size_t item_mul) {
                if (dbl) launch_wrap_fix_d(y, ST, tail, T, nitems, item_mul, nc, N, W, s);
                else launch_wrap_fix(y, ST, tail, T, nitems, item_mul, nc, N, W, cT, s);
            };
            if (comb) fix(PB, PT, np, 2);
            else fix(PB, PT, nc, 1);
            fix(QB, QT, np, 2);
            if (needR) fix(RB, RT, np, 2);
            PIC_CHECK_LAUNCH();
            count_launch(needR ? 3 : 2);
        }
        if (comb) {
            fill_u32_kernel<<<grid_for(np, 256), 256, 0, s>>>(o.l1, np, combined_words(sh, ncoef));
        } else {
            product_len_kernel<<<grid_for(np, 256), 256, 0, s>>>(ch.P.len.get(), ch.Q.len.get(), p0, np, 0, 1, o.l1);
            product_len_kernel<<<grid_for(np, 256), 256, 0, s>>>(ch.P.len.get(), ch.R.len.get(), p0, np, 1, 0, o.l2);
        }
        product_len_kernel<<<grid_for(np, 256), 256, 0, s>>>(ch.Q.len.get(), ch.Q.len.get(), p0, np, 0, 1, o.lQ);
        if (needR)
            product_len_kernel<<<grid_for(np, 256), 256, 0, s>>>(ch.R.len.get(), ch.R.len.get(), p0, np, 0, 1, o.lR);
        PIC_CHECK_LAUNCH();
        count_launch(needR ? 4 : 3);
        // T1: residues at bP items 2i (stride 2 ST), T2 at items 2i+1
        const size_t pstride = nc * ST;  // [prime][child][ST]
        auto to_words = [&](const uint64_t* y, uint32_t* z, uint32_t zcap, const uint32_t* zlen, bool offset) {
            if (dbl) ntt3d_batch_to_words(y, 2 * ST, pstride, np, k, z, zcap, zlen, s, ncoef, offset);
            else ntt3_batch_to_words(y, 2 * ST, pstride, np, k, z, zcap, zlen, s, ncoef, offset);
        };
        if (comb) {
            to_words(PB, o.T1, o.c1, o.l1, true);
        } else {
            to_words(PB, o.T1, o.c1, o.l1, false);
            to_words(PB + ST, o.T2, o.c2, o.l2, false);
        }
        to_words(QB, o.Q, o.cQ, o.lQ, false);
        if (needR) to_words(RB, o.R, o.cR, o.lR, false);
        if (!comb) {
            fix_top_kernel<<<grid_for(np, 256), 256, 0, s>>>(o.T1, o.c1, o.l1, np);
            fix_top_kernel<<<grid_for(np, 256), 256, 0, s>>>(o.T2, o.c2, o.l2, np);
        }
        fix_top_kernel<<<grid_for(np, 256), 256, 0, s>>>(o.Q, o.cQ, o.lQ, np);
        if (needR) fix_top_kernel<<<grid_for(np, 256), 256, 0, s>>>(o.R, o.cR, o.lR, np);
        PIC_CHECK_LAUNCH();
        count_launch(needR ? 4 : 3);
    }
    (void)cmax;
}

// K = sum_(j < ncoef) 2^(159 + 64 j): bit 31 of words 4 + 2 j.
__global__ void offset_words_kernel(uint32_t* K, size_t nwords)
{
    for (size_t w = blockIdx.x * (size_t)blockDim.x + threadIdx.x; w < nwords; w += (size_t)gridDim.x * blockDim.x)
        K[w] = (w >= 4 && (w & 1) == 0) ? 0x80000000u : 0u;
}

// FP64 form: K = sum_(j < ncoef) 2^(140 + 56 j); the bits are 56 apart, so a
// word holds at most one (nwords covers the last).
__global__ void offset_words56_kernel(uint32_t* K, size_t nwords)
{
    for (size_t w = blockIdx.x * (size_t)blockDim.x + threadIdx.x; w < nwords; w += (size_t)gridDim.x * blockDim.x) {
        const int64_t lo = 32 * (int64_t)w;  // bits lo .. lo + 31
        const int64_t j = lo <= 140 ? 0 : (lo - 140 + 55) / 56;
        const int64_t b = 140 + 56 * j;
        K[w] = b < lo + 32 ? 1u << (b - lo) : 0u;
    }
}

// Addend signs of P = sL (V + K) + (not sL) K: parent i at out[2i], out[2i + 1].
__global__ void sign_pair_kernel(const uint8_t* __restrict__ cs, size_t np, uint8_t* __restrict__ out)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < np; i += (size_t)gridDim.x * blockDim.x) {
        const uint8_t a = cs[2 * i] != 0 ? 1 : 0;
        out[2 * i] = a;
        out[2 * i + 1] = 1 - a;
    }
}

// P = sa A + sb B for each parent of the chunk (signs at cS[2i], cS[2i + 1]),
// into the parent slots; many CTAs per parent when parents are few and long.
static void signed_sum(const uint32_t* A, const uint32_t* lA, uint32_t cA, const uint32_t* B, const uint32_t* lB,
                       uint32_t cB, uint32_t nmax, const uint8_t* cS, size_t p0, size_t np, Level& par, cudaStream_t s)
{
    ProfScope ps(KC_LINEAR, 12.0 * (double)np * (double)nmax, s);
    const uint32_t cpp = (uint32_t)((nmax + kWideWPC - 1) / kWideWPC);
    if (g_wide_add && np < 2 * 148 && cpp > 1) {
        DevBuf<uint32_t> hd(np, s), agg(np * cpp, s), aggc(np * cpp, s);
        PIC_CUDA(cudaMemsetAsync(hd.get(), 0, 4 * np, s));
        PIC_CUDA(cudaMemsetAsync(par.P.len.get() + p0, 0, 4 * np, s));
        WideAdd w{A, lA, B, lB, cA, cB, cS, p0, par.P.w.get(), par.P.len.get(), par.P.cap, par.sign.get(), hd.get(),
                  agg.get(), aggc.get(), cpp};
        const unsigned grid = (unsigned)(np * cpp);
        wide_cmp_kernel<<<grid, 256, 0, s>>>(w);
        wide_k1_kernel<<<grid, 256, 0, s>>>(w);
        PIC_CHECK_LAUNCH();
        carry_scan_segments(agg.get(), np, cpp, s);
        wide_ripple_kernel<<<grid, 256, 0, s>>>(w);
        wide_final_kernel<<<grid, 256, 0, s>>>(w);
        PIC_CHECK_LAUNCH();
        count_launch(4);
    } else {
        signed_add_kernel<<<(unsigned)np, 256, 0, s>>>(A, lA, cA, B, lB, cB, cS, p0, par.P.w.get(), par.P.len.get(),
                                                      par.sign.get(), par.P.cap);
        PIC_CHECK_LAUNCH();
        count_launch();
    }
}

static bool g_combine = true;  // P formed in the transform domain (one inverse, one CRT)

// Device bytes the transforms of one batch of merges may take: a quarter of
// what the device has left, at most 128 bytes per word of the precision p
// (12 GB at 1e9 digits; larger batches save little: 0.5 % of the run at
// twice the size), at least 1 GiB.  Keeping the peak proportional to p lets
// the pool reserved up front (reserve_pool, 512 bytes per word) hold every
// call without growing, the top levels' workspace included; at 256 bytes
// per word the peak outgrew it and runs stalled on pool growth.
static size_t merge_budget(size_t p)
{
    size_t b = device_available_bytes() / 4;
    b = std::min(b, p * 128);
    return std::max(b, (size_t)1 << 30);
}

static void merge_ntt(Level& ch, Level& par, cudaStream_t s, size_t mem_budget)
{
    const uint32_t ccP = ch.P.cap, ccQ = ch.Q.cap, ccR = ch.R.cap;
    const uint32_t cmax = std::max(ccP, std::max(ccQ, ccR));
    const MergeShape sh = merge_shape(cmax);
    const size_t ncoef = products_ncoef(sh);
    count_products(4 * par.count);  // P0 Q1, P1 R0, Q0 Q1, R0 R1 per parent (PI.h:110-112)
    // combined form: P = sL (T1 +- T2) converted once as V + K (the CRT adds
    // 2^159, in the FP64 form 2^140, to every coefficient so the signed ones
    // stay exact), then
    // P = sL (V + K) - sL K with the exact signed sum
    const uint32_t cV = combined_words(sh, ncoef) + 2, cK = offset_words(sh, ncoef);
    const uint32_t c1 = g_combine ? cV : ccP + ccQ, c2 = g_combine ? 0 : ccP + ccR;
    // bytes per parent: the transforms plus the word buffers for P
    const size_t per_parent = ntt_bytes_per_parent(sh) + 4 * (size_t)(c1 + c2 + ccQ + ccR);
    size_t chunk = mem_budget / per_parent;
    if (chunk < 1) chunk = 1;
    if (chunk > par.count) chunk = par.count;
    DevBuf<uint32_t> K(g_combine ? cK : 0, s);
    if (g_combine) {
        if (sh.form == kFormDbl) offset_words56_kernel<<<grid_for(cK, 256), 256, 0, s>>>(K.get(), cK);
        else offset_words_kernel<<<grid_for(cK, 256), 256, 0, s>>>(K.get(), cK);
        PIC_CHECK_LAUNCH();
        count_launch();
    }
    for (size_t p0 = 0; p0 < par.count; p0 += chunk) {
        const size_t np = std::min(chunk, par.count - p0);
        DevBuf<uint32_t> T1(np * c1, s), T2(g_combine ? 0 : np * c2, s), l1(np, s), l2(np, s);
        ProductsOut o;
        o.T1 = T1.get();
        o.c1 = c1;
        o.l1 = l1.get();
        o.T2 = T2.get();
        o.c2 = c2;
        o.l2 = l2.get();
        o.Q = par.Q.w.get() + p0 * par.Q.cap;
        o.cQ = par.Q.cap;
        o.lQ = par.Q.len.get() + p0;
        o.R = par.R.w.get() + p0 * par.R.cap;
        o.cR = par.R.cap;
        o.lR = par.R.len.get() + p0;
        if (g_combine) o.csign = ch.sign.get() + 2 * p0;
        ntt_products(ch, p0, np, sh, o, s);
        if (g_combine) {
            DevBuf<uint8_t> sg(2 * np, s);
            sign_pair_kernel<<<grid_for(np, 256), 256, 0, s>>>(ch.sign.get() + 2 * p0, np, sg.get());
            fill_u32_kernel<<<grid_for(np, 256), 256, 0, s>>>(l2.get(), np, cK);
            PIC_CHECK_LAUNCH();
            count_launch(2);
            signed_sum(T1.get(), l1.get(), c1, K.get(), l2.get(), 0, cV, sg.get(), p0, np, par, s);
        } else {
            signed_sum(T1.get(), l1.get(), c1, T2.get(), l2.get(), c2, std::max(c1, c2), ch.sign.get() + 2 * p0, p0,
                       np, par, s);
        }
    }
}

static void merge_school(Level& ch, Level& par, cudaStream_t s)
{
    MergeArgs m;
    m.cPw = ch.P.w.get();
    m.cQw = ch.Q.w.get();
    m.cRw = ch.R.w.get();
    m.cPl = ch.P.len.get();
    m.cQl = ch.Q.len.get();
    m.cRl = ch.R.len.get();
    m.cS = ch.sign.get();
    m.ccP = ch.P.cap;
    m.ccQ = ch.Q.cap;
    m.ccR = ch.R.cap;
    m.pPw = par.P.w.get();
    m.pQw = par.Q.w.get();
    m.pRw = par.R.w.get();
    m.pPl = par.P.len.get();
    m.pQl = par.Q.len.get();
    m.pRl = par.R.len.get();
    m.pS = par.sign.get();
    m.pcP = par.P.cap;
    m.pcQ = par.Q.cap;
    m.pcR = par.R.cap;
    m.count = par.count;
    m.kara_min = g_kara_min;
    const size_t words = 2 * ((size_t)m.ccP + m.ccQ + m.ccR) + (m.ccP + m.ccQ) + (m.ccP + m.ccR) +
                         3 * ((size_t)m.ccP + m.ccQ) + (g_kara_min ? 3 * ((size_t)m.ccP + m.ccQ) + 8 : 0);
    const size_t smem = words * sizeof(uint32_t);
    PIC_REQUIRE(smem <= 200 * 1024, PIC_ERR_INVALID, "schoolbook merge tile too large");
    if (smem > 48 * 1024)
        PIC_CUDA(cudaFuncSetAttribute(merge_school_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const uint32_t cmax = std::max(m.ccP, std::max(m.ccQ, m.ccR));
    count_products(4 * par.count);  // P0 Q1, P1 R0, Q0 Q1, R0 R1 per parent (PI.h:110-112)
    ProfScope ps(KC_BSR, 4.0 * (double)par.count * 2.0 * (m.ccP + m.ccQ + m.ccR), s);
    if (g_small_merge >= 2 && (launch_merge_thread<16, 16, 12>(m, s) || launch_merge_thread<20, 20, 14>(m, s) ||
                               launch_merge_thread<28, 28, 20>(m, s))) {
        PIC_CHECK_LAUNCH();
        count_launch();
        return;
    }
    if (cmax <= (uint32_t)kWarpMergeMax && g_small_merge >= 1) {
        const size_t wsmem = sizeof(uint32_t) * warp_merge_words(m.ccP, m.ccQ, m.ccR) * kWarpMergeWarps;
        if (wsmem > 48 * 1024)
            PIC_CUDA(cudaFuncSetAttribute(merge_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wsmem));
        const size_t grid = (par.count + kWarpMergeWarps - 1) / kWarpMergeWarps;
        merge_warp_kernel<<<(unsigned)grid, 32 * kWarpMergeWarps, wsmem, s>>>(m);
        PIC_CHECK_LAUNCH();
        count_launch();
        return;
    }
    const int threads = cmax <= 16 ? 32 : (cmax <= 64 ? 64 : (cmax <= 256 ? 128 : 256));
    merge_school_kernel<<<(unsigned)par.count, threads, smem, s>>>(m);
    PIC_CHECK_LAUNCH();
    count_launch();
}

// Largest child capacity handled by the CTA schoolbook merge.
static uint32_t g_school_max = 600;

void bsr_set_school_threshold(uint32_t words) { g_school_max = words; }
void bsr_set_wrap(bool on) { g_wrap = on; }
void bsr_set_karatsuba(uint32_t min_words) { g_kara_min = min_words; }
uint32_t bsr_karatsuba() { return g_kara_min; }
void bsr_set_combine(bool on) { g_combine = on; }
bool bsr_combine() { return g_combine; }
void bsr_set_small_merge(int mode) { g_small_merge = mode; }
int bsr_small_merge() { return g_small_merge; }
bool bsr_wrap() { return g_wrap; }
uint32_t bsr_school_threshold() { return g_school_max; }

static void alloc_level(Level& L, size_t count, uint32_t cP, uint32_t cQ, uint32_t cR, cudaStream_t s)
{
    L.count = count;
    alloc_slots(L.P, count, cP, s);
    alloc_slots(L.Q, count, cQ, s);
    alloc_slots(L.R, count, cR, s);
    L.sign = DevBuf<uint8_t>(count, s);
}

// Recursion above the batched depth, exactly the reference's merges with
// truncation (PI.h:93-112); nodes at `stop_depth` come from `top`.
struct TopSource {
    std::vector<BigFloat> P, Q, R;
    size_t next = 0;
};

static void bsr_top(BigFloat& P, BigFloat& Q, BigFloat& R, uint32_t a, uint32_t b, size_t p, int depth,
                    int stop_depth, TopSource& src, bool need_R = true)
{
    if (depth == stop_depth) {
        P = src.P[src.next];
        Q = src.Q[src.next];
        R = src.R[src.next];
        src.next++;
        return;
    }
    if (b - a == 1) {  // only reached when the whole tree is shallower than stop_depth
        bsr_recursive(P, Q, R, a, b, p);
        return;
    }
    const uint32_t m = (a + b) / 2;
    BigFloat P0, Q0, R0, P1, Q1, R1;
    bsr_top(P0, Q0, R0, a, m, p, depth + 1, stop_depth, src);
    bsr_top(P1, Q1, R1, m, b, p, depth + 1, stop_depth, src);
    P = P0.mul(Q1, p).add(P1.mul(R0, p), p);
    Q = Q0.mul(Q1, p);
    if (need_R) R = R0.mul(R1, p);
}

// One level of the merges above the batched range, the reference's merge with
// precision p (PI.h:110-112): every operand is chopped to its top p + 2 words
// as BigFloat::mul does (BigFloat.cpp:337-366), the four products are exact
// products of the chopped operands computed together (each operand
// transformed once, wrapped lengths), and P = T1.add(T2, p) with the
// reference's add.  Children 2i, 2i + 1 -> parent i.  Returns false (and
// computes nothing) if a Q or R child is negative, which the series never
// produces.
static bool top_level_merge(const std::vector<BigFloat>& cP, const std::vector<BigFloat>& cQ,
                            const std::vector<BigFloat>& cR, size_t p, bool need_R, std::vector<BigFloat>& oP,
                            std::vector<BigFloat>& oQ, std::vector<BigFloat>& oR, cudaStream_t s)
{
    const size_t nc = cP.size(), np = nc / 2;
    trace_point("top_merge_begin", s);
    timeline_mark("top_merge_begin", s);
    struct View {
        const uint32_t* T;
        size_t L;
        int64_t exp;
        bool sign;
    };
    const size_t pw = p + 2;  // p + YCL_BIGFLOAT_EXTRA_PRECISION (BigFloat.h:6)
    auto chop = [&](const BigFloat& x) {
        View v{x.device_words(), x.get_precision(), x.get_exponent(), x.get_sign()};
        if (p != 0 && v.L > pw) {
            const size_t c = v.L - pw;
            v.T += c;
            v.L = pw;
            v.exp += (int64_t)c;
        }
        return v;
    };
    std::vector<View> vP(nc), vQ(nc), vR(nc);
    uint32_t capP = 1, capQ = 1, capR = 1;
    for (size_t i = 0; i < nc; i++) {
        vP[i] = chop(cP[i]);
        vQ[i] = chop(cQ[i]);
        vR[i] = chop(cR[i]);
        if (!vQ[i].sign || !vR[i].sign) return false;
        capP = std::max<uint32_t>(capP, (uint32_t)vP[i].L);
        capQ = std::max<uint32_t>(capQ, (uint32_t)vQ[i].L);
        capR = std::max<uint32_t>(capR, (uint32_t)vR[i].L);
    }
    // the children as a batched level
    Level ch;
    alloc_level(ch, nc, capP, capQ, capR, s);
    std::vector<uint32_t> lP(nc), lQ(nc), lR(nc);
    std::vector<uint8_t> sg(nc);
    for (size_t i = 0; i < nc; i++) {
        if (vP[i].L)
            PIC_CUDA(cudaMemcpyAsync(ch.P.w.get() + i * capP, vP[i].T, 4 * vP[i].L, cudaMemcpyDeviceToDevice, s));
        if (vQ[i].L)
            PIC_CUDA(cudaMemcpyAsync(ch.Q.w.get() + i * capQ, vQ[i].T, 4 * vQ[i].L, cudaMemcpyDeviceToDevice, s));
        if (vR[i].L)
            PIC_CUDA(cudaMemcpyAsync(ch.R.w.get() + i * capR, vR[i].T, 4 * vR[i].L, cudaMemcpyDeviceToDevice, s));
        lP[i] = (uint32_t)vP[i].L;
        lQ[i] = (uint32_t)vQ[i].L;
        lR[i] = (uint32_t)vR[i].L;
        sg[i] = vP[i].sign ? 1 : 0;
    }
    PIC_CUDA(cudaMemcpyAsync(ch.P.len.get(), lP.data(), 4 * nc, cudaMemcpyHostToDevice, s));
    PIC_CUDA(cudaMemcpyAsync(ch.Q.len.get(), lQ.data(), 4 * nc, cudaMemcpyHostToDevice, s));
    PIC_CUDA(cudaMemcpyAsync(ch.R.len.get(), lR.data(), 4 * nc, cudaMemcpyHostToDevice, s));
    PIC_CUDA(cudaMemcpyAsync(ch.sign.get(), sg.data(), nc, cudaMemcpyHostToDevice, s));
    trace_point("top_merge_children", s);
    timeline_mark("top_merge_children", s);
    // the products, in parent chunks that fit a quarter of the free memory
    const MergeShape sh = merge_shape(std::max(capP, std::max(capQ, capR)));
    const uint32_t c1 = capP + capQ, c2 = capP + capR, cq = 2 * capQ, cr = 2 * capR;
    auto sT1 = alloc_words(np * c1), sT2 = alloc_words(np * c2), sQ = alloc_words(np * cq);
    std::shared_ptr<WordStore> sR = need_R ? alloc_words(np * cr) : nullptr;
    DevBuf<uint32_t> lens(4 * np, s);
    count_products((need_R ? 4 : 3) * np);
    size_t chunk = merge_budget(p) / ntt_bytes_per_parent(sh);
    if (chunk < 1) chunk = 1;
    for (size_t p0 = 0; p0 < np; p0 += chunk) {
        const size_t n = std::min(chunk, np - p0);
        ProductsOut o;
        o.T1 = sT1->base + p0 * c1;
        o.c1 = c1;
        o.l1 = lens.get() + p0;
        o.T2 = sT2->base + p0 * c2;
        o.c2 = c2;
        o.l2 = lens.get() + np + p0;
        o.Q = sQ->base + p0 * cq;
        o.cQ = cq;
        o.lQ = lens.get() + 2 * np + p0;
        if (need_R) {
            o.R = sR->base + p0 * cr;
            o.cR = cr;
            o.lR = lens.get() + 3 * np + p0;
        }
        ntt_products(ch, p0, n, sh, o, s, /*use_workspace=*/true);
        trace_point("top_merge_chunk", s);
        timeline_mark("top_merge_chunk", s, sh.k);
    }
    std::vector<uint32_t> hl(4 * np, 0);
    PIC_CUDA(cudaMemcpyAsync(hl.data(), lens.get(), 4 * (need_R ? 4 : 3) * np, cudaMemcpyDeviceToHost, s));
    PIC_CUDA(cudaStreamSynchronize(s));
    // BigFloat::mul's result: sign product, exponent sum, empty if an operand is
    auto product = [&](const View& x, const View& y, const std::shared_ptr<WordStore>& st, const uint32_t* w,
                       uint32_t L) {
        if (x.L == 0 || y.L == 0) return BigFloat();
        return BigFloat::from_device(x.sign == y.sign, x.exp + y.exp, st, w, L);
    };
    oP.resize(np);
    oQ.resize(np);
    oR.resize(np);
    for (size_t i = 0; i < np; i++) {
        const size_t L = 2 * i, R = 2 * i + 1;
        const BigFloat t1 = product(vP[L], vQ[R], sT1, sT1->base + i * c1, hl[i]);
        const BigFloat t2 = product(vP[R], vR[L], sT2, sT2->base + i * c2, hl[np + i]);
        oP[i] = t1.add(t2, p);
        oQ[i] = product(vQ[L], vQ[R], sQ, sQ->base + i * cq, hl[2 * np + i]);
        oR[i] = need_R ? product(vR[L], vR[R], sR, sR->base + i * cr, hl[3 * np + i]) : BigFloat();
    }
    trace_point("top_merge_adds", s);
    timeline_mark("top_merge_adds", s);
    return true;
}

void bsr_chosen(BigFloat& P, BigFloat& Q, BigFloat& R, uint32_t a, uint32_t b, size_t p, bool need_root_R)
{
    cudaStream_t s = ctx().stream;
    const uint32_t T = b - a;
    // bottom depth: node lengths <= 2
    int Db = 0;
    while ((((uint64_t)T + ((1ull << Db) - 1)) >> Db) > 2) Db++;
    // top of the batched range: the shallowest depth whose merges cannot truncate
    // (every operand <= p + 2 words and every add window <= p + 2)
    int Dtop = Db;
    for (int d = Db - 1; d >= 0; d--) {
        const double nchild = ceil((double)T / (double)(1ull << (d + 1)));
        uint32_t cP, cQ, cR;
        slot_caps(nchild, (double)b, cP, cQ, cR);
        if ((size_t)cP + cQ > p + 2 || (size_t)cP + cR > p + 2) break;
        Dtop = d;
    }
    // the bottom kernel merges pairs of leaves exactly: that needs the
    // reference's p + 2 window to hold two leaves (<= 6 + 5 words)
    if (p < 16 || T < 4) {
        bsr_recursive(P, Q, R, a, b, p);
        return;
    }
    // boundaries, top down
    std::vector<DevBuf<uint32_t>> bnd(Db + 1);
    {
        bnd[0] = DevBuf<uint32_t>(2, s);
        const uint32_t h[2] = {a, b};
        PIC_CUDA(cudaMemcpyAsync(bnd[0].get(), h, sizeof h, cudaMemcpyHostToDevice, s));
        PIC_CUDA(cudaStreamSynchronize(s));
        for (int d = 0; d < Db; d++) {
            const size_t cnt = (size_t)1 << d;
            bnd[d + 1] = DevBuf<uint32_t>(2 * cnt + 1, s);
            split_bounds_kernel<<<grid_for(cnt, 256), 256, 0, s>>>(bnd[d].get(), cnt, bnd[d + 1].get());
            PIC_CHECK_LAUNCH();
            count_launch();
        }
    }
    timeline_mark("bsr_bounds", s);
    // bottom level
    Level cur;
    {
        const size_t cnt = (size_t)1 << Db;
        uint32_t cP, cQ, cR;
        slot_caps(2.0, (double)b, cP, cQ, cR);
        cP = std::max(cP, 12u);
        cQ = std::max(cQ, 10u);
        cR = std::max(cR, 8u);
        alloc_level(cur, cnt, cP, cQ, cR, s);
        ProfScope ps(KC_BSR, (double)cnt * 4.0 * (cP + cQ + cR), s);
        bottom_kernel<<<grid_for(cnt, 128), 128, 0, s>>>(bnd[Db].get(), cnt, cur.P.w.get(), cur.P.len.get(),
                                                         cur.sign.get(), cP, cur.Q.w.get(), cur.Q.len.get(), cQ,
                                                         cur.R.w.get(), cur.R.len.get(), cR);
        PIC_CHECK_LAUNCH();
        count_launch();
    }
    timeline_mark("bsr_bottom", s);
    // merge up to Dtop
    const size_t budget = merge_budget(p);
    for (int d = Db - 1; d >= Dtop; d--) {
        const size_t cnt = (size_t)1 << d;
        const double n = ceil((double)T / (double)cnt);
        uint32_t cP, cQ, cR;
        slot_caps(n, (double)b, cP, cQ, cR);
        Level par;
        alloc_level(par, cnt, cP, cQ, cR, s);
        const uint32_t cmax = std::max(cur.P.cap, std::max(cur.Q.cap, cur.R.cap));
        TraceSpan span(s);
        const bool school = cmax <= g_school_max;
        if (school) merge_school(cur, par, s);
        else merge_ntt(cur, par, s, budget);
        if (tracing())
            fprintf(stderr,
                    "{\"trace\": \"bsr_level\", \"depth\": %d, \"parents\": %zu, \"child_caps\": [%u, %u, %u], "
                    "\"algo\": \"%s\", \"ms\": %.3f}\n",
                    d, cnt, cur.P.cap, cur.Q.cap, cur.R.cap, school ? "school" : "ntt3", span.end_ms());
        cur = std::move(par);
        bnd[d + 1].reset();
        timeline_mark(school ? "bsr_level_school" : "bsr_level_ntt", s, school ? -1 : merge_shape(cmax).k);
    }
    // hand the nodes at Dtop to the exact BigFloat recursion
    const size_t cnt = cur.count;
    std::vector<uint32_t> lP(cnt), lQ(cnt), lR(cnt);
    std::vector<uint8_t> sg(cnt);
    PIC_CUDA(cudaMemcpyAsync(lP.data(), cur.P.len.get(), cnt * 4, cudaMemcpyDeviceToHost, s));
    PIC_CUDA(cudaMemcpyAsync(lQ.data(), cur.Q.len.get(), cnt * 4, cudaMemcpyDeviceToHost, s));
    PIC_CUDA(cudaMemcpyAsync(lR.data(), cur.R.len.get(), cnt * 4, cudaMemcpyDeviceToHost, s));
    PIC_CUDA(cudaMemcpyAsync(sg.data(), cur.sign.get(), cnt, cudaMemcpyDeviceToHost, s));
    PIC_CUDA(cudaStreamSynchronize(s));
    auto own = [&](Slots& sl) {
        auto st = std::make_shared<WordStore>();
        st->base = sl.w.ptr;
        st->bytes = sizeof(uint32_t) * (sl.w.n ? sl.w.n : 1);
        sl.w.ptr = nullptr;  // ownership moves to the WordStore
        sl.w.n = 0;
        return st;
    };
    auto sP = own(cur.P), sQ = own(cur.Q), sR = own(cur.R);
    TopSource src;
    src.P.reserve(cnt);
    for (size_t i = 0; i < cnt; i++) {
        src.P.push_back(BigFloat::from_device(sg[i] != 0, 0, sP, sP->base + i * cur.P.cap, lP[i]));
        src.Q.push_back(BigFloat::from_device(true, 0, sQ, sQ->base + i * cur.Q.cap, lQ[i]));
        src.R.push_back(BigFloat::from_device(true, 0, sR, sR->base + i * cur.R.cap, lR[i]));
    }
    TraceSpan tspan(s);
    // levels Dtop - 1 .. 0, each as one batched merge of all its parents;
    // `stop` is the depth the node lists in src hold
    int stop = Dtop;
    for (int d = Dtop - 1; d >= 0 && g_top_batched; d--) {
        std::vector<BigFloat> nP, nQ, nR;
        TraceSpan lspan(s);
        if (!top_level_merge(src.P, src.Q, src.R, p, d > 0 || need_root_R, nP, nQ, nR, s)) break;
        if (tracing())
            fprintf(stderr, "{\"trace\": \"bsr_top_level\", \"depth\": %d, \"parents\": %zu, \"ms\": %.3f}\n", d,
                    nP.size(), lspan.end_ms());
        src.P = std::move(nP);
        src.Q = std::move(nQ);
        src.R = std::move(nR);
        stop = d;
    }
    if (stop == 0) {
        P = src.P[0];
        Q = src.Q[0];
        R = src.R[0];
    } else {
        src.next = 0;
        bsr_top(P, Q, R, a, b, p, 0, stop, src, need_root_R);
    }
    if (tracing())
        fprintf(stderr, "{\"trace\": \"bsr_top\", \"nodes\": %zu, \"depth\": %d, \"ms\": %.3f}\n", cnt, Dtop,
                tspan.end_ms());
}

}  // namespace pic
