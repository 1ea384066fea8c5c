// NTT engine kernels and twiddle tables (see ntt.cuh for the layout).
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <tuple>
#include <vector>
#include <mutex>
#include <type_traits>

#include "common.cuh"
#include "fp64mod.cuh"
#include "ntt.cuh"

namespace pic {

// Three primes c * 2^32 + 1 between 2^64 / 9 and 2^61 (2-adicity 32, 33,
// 33); their product is ~2^183, so a cyclic convolution of 64-bit pieces of
// length <= 2^30 (any coefficient < 2^158, or a signed difference of two such)
// is recovered exactly by CRT.  Below 2^61, 8p < 2^64 leaves room for lazy
// residues in [0, 4p) (forward) and [0, 8p) (inverse) and for the
// three-partial-product Shoup quotient; above 2^64 / 9 a 64-bit piece is below
// 9p and reaches [0, 4p) with two conditional subtractions.
const uint64_t kProductPrimes[3] = {2305842979148922881ull, 2305842949084151809ull,
                                    2305842811645198337ull};

// Three primes c * 2^32 + 1 just below 2^47 (2-adicity 35, 32, 32), the FP64
// product form's: their product is ~2^140.99, so a convolution of 56-bit
// pieces whose shorter operand has at most 2^28 pieces (coefficients below
// 2^140) is recovered exactly, and with the offset 2^140 so is a signed sum
// of two products of at most 2^26 pieces (the merges' limit; at 2^27 the
// worst case would pass the primes' product).  Below 2^47, forward values up to
// 16 p stay under 2^51, the range of the FP64 quotient.
const uint64_t kDblPrimes[3] = {140496970186753ull, 140458315481089ull, 140449725546497ull};

// The reference's prime table, NTT.cpp:125-158.  The transform length picks
// the prime, so natural-order outputs only match if the values match.
static const uint64_t k_ref_primes[43] = {
    0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0,
    9223372036854675457ull, 9223372036854497281ull, 9223372036854497281ull,
    9223372036854497281ull, 9223372036853661697ull, 9223372036853661697ull,
    9223372036844421121ull, 9223372036836950017ull, 9223372036836950017ull,
    9223372036836950017ull, 9223372036752015361ull, 9223372036737335297ull,
    9223372036737335297ull, 9223372036737335297ull, 9223372036083023873ull,
    9223372035915251713ull, 9223372035915251713ull, 9223372034170421249ull,
    9223372034170421249ull, 9223372006790004737ull, 9223372006790004737ull,
    9223372006790004737ull, 9223371564408373249ull, 9223371280940531713ull,
    9223371280940531713ull, 9223371280940531713ull, 9223369837831520257ull,
    9223369837831520257ull, 9223369837831520257ull, 9223369837831520257ull,
    9223369837831520257ull, 9223341250529198081ull};

uint64_t reference_prime(int k)
{
    if (k < 11) k = 11;
    if (k > 42) return 0;
    return k_ref_primes[k];
}

// NTT.cpp:104-123: factor p-1 by trial division, then the smallest g >= 2
// with g^((p-1)/q) != 1 for every prime factor q.
uint64_t smallest_generator(uint64_t p)
{
    uint64_t fact[64];
    int nf = 0;
    uint64_t phi = p - 1, n = phi;
    for (uint64_t i = 2; i * i <= n; ++i)
        if (n % i == 0) {
            fact[nf++] = i;
            while (n % i == 0) n /= i;
        }
    if (n > 1) fact[nf++] = n;
    for (uint64_t g = 2; g <= p; ++g) {
        bool ok = true;
        for (int i = 0; i < nf && ok; ++i) ok = host_powmod(g, phi / fact[i], p) != 1;
        if (ok) return g;
    }
    return 0;
}

static std::mutex g_tab_lock;
static std::map<uint64_t, PrimeTables*> g_tabs;

static uint64_t* upload(const std::vector<uint64_t>& v)
{
    uint64_t* d = nullptr;
    PIC_CUDA(raw_dev_alloc((void**)&d, v.size() * sizeof(uint64_t)));
    PIC_CUDA(cudaMemcpy(d, v.data(), v.size() * sizeof(uint64_t), cudaMemcpyHostToDevice));
    return d;
}

const PrimeTables& prime_tables(uint64_t p)
{
    std::lock_guard<std::mutex> g(g_tab_lock);
    auto it = g_tabs.find(p);
    if (it != g_tabs.end()) return *it->second;
    PrimeTables* t = new PrimeTables();
    t->p = p;
    t->g = smallest_generator(p);
    int v = 0;
    while (((p - 1) >> v & 1) == 0) v++;
    t->adicity = v;
    const int K = v < 32 ? v : 32;
    const int S = (K + 1) / 2;
    const int IB = K < kInnerBits ? K : kInnerBits;
    const Mod64 m = make_mod(p);
    const uint64_t wK = host_powmod(t->g, (p - 1) >> K, p);
    const uint64_t wKi = host_powmod(wK, p - 2, p);

    std::vector<uint64_t> inf((size_t)2 << (IB - 1)), ini((size_t)2 << (IB - 1));
    const uint64_t wI = host_powmod(wK, (uint64_t)1 << (K - IB), p);
    const uint64_t wIi = host_powmod(wKi, (uint64_t)1 << (K - IB), p);
    uint64_t a = 1, b = 1;
    for (size_t i = 0; i < ((size_t)1 << (IB - 1)); i++) {
        inf[2 * i] = a;
        inf[2 * i + 1] = shoup_companion(a, p);
        ini[2 * i] = b;
        ini[2 * i + 1] = shoup_companion(b, p);
        a = host_mulmod(a, wI, p);
        b = host_mulmod(b, wIi, p);
    }
    std::vector<uint64_t> lof((size_t)1 << S), loi((size_t)1 << S);
    std::vector<uint64_t> hif((size_t)1 << (K - S)), hii((size_t)1 << (K - S));
    a = 1, b = 1;
    for (size_t i = 0; i < lof.size(); i++) {
        lof[i] = to_mont(a, p);
        loi[i] = to_mont(b, p);
        a = host_mulmod(a, wK, p);
        b = host_mulmod(b, wKi, p);
    }
    const uint64_t wS = a, wSi = b;  // root^(2^S)
    a = 1, b = 1;
    for (size_t i = 0; i < hif.size(); i++) {
        hif[i] = to_mont(a, p);
        hii[i] = to_mont(b, p);
        a = host_mulmod(a, wS, p);
        b = host_mulmod(b, wSi, p);
    }
    PrimeDev& d = t->dev;
    d.p = p;
    d.pinv_neg = m.pinv_neg;
    d.r2 = m.r2;
    d.K = K;
    d.S = S;
    d.IB = IB;
    // lazy butterflies need 8p < 2^64 and the c * 2^32 + 1 form (mul_p_lo)
    d.lazy = (p < (1ull << 61) && (p & 0xffffffffull) == 1) ? 1 : 0;
    {
        const unsigned __int128 mu = (~(unsigned __int128)0) / p;  // floor(2^128 / p): p does not divide 2^128
        d.mu_hi = (uint64_t)(mu >> 64);
        d.mu_lo = (uint64_t)mu;
    }
    d.inner_fwd = upload(inf);
    d.inner_inv = upload(ini);
    d.olo_fwd = upload(lof);
    d.ohi_fwd = upload(hif);
    d.olo_inv = upload(loi);
    d.ohi_inv = upload(hii);
    if (d.lazy) {
        // the same outer roots as Shoup pairs (plain value, companion)
        auto pairs = [&](const std::vector<uint64_t>& mont) {
            std::vector<uint64_t> v(2 * mont.size());
            const uint64_t rinv = host_powmod(to_mont(1, p), p - 2, p);  // R^-1 mod p
            for (size_t i = 0; i < mont.size(); i++) {
                const uint64_t x = host_mulmod(mont[i], rinv, p);
                v[2 * i] = x;
                v[2 * i + 1] = shoup_companion(x, p);
            }
            return upload(v);
        };
        d.slo_fwd = pairs(lof);
        d.shi_fwd = pairs(hif);
        d.slo_inv = pairs(loi);
        d.shi_inv = pairs(hii);
        if (IB == kInnerBits) {
            // per-level inner tables from the order-2^IB tables: the root of
            // order 2^m is inner root^(2^(IB - m))
            std::vector<uint64_t> lf((size_t)2 << IB), li((size_t)2 << IB);
            for (int lm = 1; lm <= IB; lm++)
                for (size_t e = 0; e < ((size_t)1 << (lm - 1)); e++) {
                    const size_t dst = ((size_t)1 << (lm - 1)) - 1 + e, src = e << (IB - lm);
                    lf[2 * dst] = inf[2 * src];
                    lf[2 * dst + 1] = inf[2 * src + 1];
                    li[2 * dst] = ini[2 * src];
                    li[2 * dst + 1] = ini[2 * src + 1];
                }
            d.lvl_fwd = upload(lf);
            d.lvl_inv = upload(li);
        }
    }
    g_tabs[p] = t;
    return *t;
}

// An FP64 table entry: w as a double (the companion fl(w fl(1 / p)) is formed
// where the twiddle is used).
static void dbl_entry(std::vector<uint64_t>& v, size_t i, uint64_t w)
{
    const double wd = (double)w;
    memcpy(&v[i], &wd, 8);
}

const PrimeTables& dbl_prime_tables(uint64_t p)
{
    PIC_REQUIRE(p < (1ull << 47) && p > (1ull << 40), PIC_ERR_INVALID, "FP64 primes lie in (2^40, 2^47)");
    std::lock_guard<std::mutex> g(g_tab_lock);
    auto it = g_tabs.find(p);
    if (it != g_tabs.end()) return *it->second;
    PrimeTables* t = new PrimeTables();
    t->p = p;
    t->g = smallest_generator(p);
    int v = 0;
    while (((p - 1) >> v & 1) == 0) v++;
    t->adicity = v;
    PIC_REQUIRE(v >= kInnerBits, PIC_ERR_INVALID, "FP64 prime without roots of order 2^13");
    const int K = v < 32 ? v : 32;
    const int S = (K + 1) / 2;
    const int IB = kInnerBits;
    const uint64_t wK = host_powmod(t->g, (p - 1) >> K, p);
    const uint64_t wKi = host_powmod(wK, p - 2, p);
    const uint64_t wI = host_powmod(wK, (uint64_t)1 << (K - IB), p);
    const uint64_t wIi = host_powmod(wKi, (uint64_t)1 << (K - IB), p);
    // per-level inner tables: the root of order 2^m is wI^(2^(IB - m)); pair
    // 2^(m-1) - 1 + e holds its e-th power
    std::vector<uint64_t> lf((size_t)1 << IB), li((size_t)1 << IB);
    for (int lm = 1; lm <= IB; lm++) {
        const uint64_t r = host_powmod(wI, (uint64_t)1 << (IB - lm), p);
        const uint64_t ri = host_powmod(wIi, (uint64_t)1 << (IB - lm), p);
        uint64_t a = 1, b = 1;
        for (size_t e = 0; e < ((size_t)1 << (lm - 1)); e++) {
            const size_t dst = ((size_t)1 << (lm - 1)) - 1 + e;
            dbl_entry(lf, dst, a);
            dbl_entry(li, dst, b);
            a = host_mulmod(a, r, p);
            b = host_mulmod(b, ri, p);
        }
    }
    // two-level outer tables: root_(2^K)^i (i < 2^S) and root_(2^K)^(i 2^S)
    std::vector<uint64_t> lof((size_t)1 << S), loi((size_t)1 << S);
    std::vector<uint64_t> hif((size_t)1 << (K - S)), hii((size_t)1 << (K - S));
    uint64_t a = 1, b = 1;
    for (size_t i = 0; i < ((size_t)1 << S); i++) {
        dbl_entry(lof, i, a);
        dbl_entry(loi, i, b);
        a = host_mulmod(a, wK, p);
        b = host_mulmod(b, wKi, p);
    }
    const uint64_t wS = a, wSi = b;
    a = 1, b = 1;
    for (size_t i = 0; i < ((size_t)1 << (K - S)); i++) {
        dbl_entry(hif, i, a);
        dbl_entry(hii, i, b);
        a = host_mulmod(a, wS, p);
        b = host_mulmod(b, wSi, p);
    }
    PrimeDev& d = t->dev;
    memset(&d, 0, sizeof d);
    d.p = p;
    d.K = K;
    d.S = S;
    d.IB = IB;
    d.lazy = 0;
    d.fp64 = 1;
    d.pd = (double)p;
    d.pinv = 1.0 / (double)p;
    d.slo_fwd = upload(lof);
    d.shi_fwd = upload(hif);
    d.slo_inv = upload(loi);
    d.shi_inv = upload(hii);
    d.lvl_fwd = upload(lf);
    d.lvl_inv = upload(li);
    g_tabs[p] = t;
    return *t;
}

// Per-length geometry (tunable; pic_set_ntt_geometry): row-pass bits, column
// tile width (log2 columns per CTA, 0 = automatic) and bits per register round
// (radix 2^rbits).
struct Geometry {
    int row_bits = 12;
    int col_lw = 0;
    int rbits = 3;
};
static Geometry g_geom_forms[2][33];

static const Geometry& geom_of(const NttBatch& b, int k) { return g_geom_forms[b.prime[0].fp64 ? 1 : 0][k]; }

void ntt_set_geometry(int k, int row_bits, int col_lw, int rbits, int form)
{
    PIC_REQUIRE(form == kFormInt || form == kFormDbl, PIC_ERR_INVALID, "unknown product form");
    PIC_REQUIRE(k >= 1 && k <= 32, PIC_ERR_INVALID, "k out of range");
    PIC_REQUIRE(row_bits >= (form == kFormDbl ? 11 : 8) && row_bits <= kInnerBits, PIC_ERR_INVALID,
                "row bits out of range (8..13; FP64 form 11..13)");
    PIC_REQUIRE(col_lw >= 0 && col_lw <= 6, PIC_ERR_INVALID, "column width out of range (0..6)");
    PIC_REQUIRE(rbits >= (form == kFormDbl ? 3 : 2) && rbits <= 4, PIC_ERR_INVALID,
                "radix bits out of range (2..4; FP64 form 3..4)");
    Geometry& g = g_geom_forms[form][k];
    g.row_bits = row_bits;
    g.col_lw = col_lw;
    g.rbits = rbits;
}

void ntt_get_geometry(int k, int* row_bits, int* col_lw, int* rbits, int form)
{
    const Geometry& g = g_geom_forms[form == kFormDbl ? 1 : 0][k < 1 ? 1 : (k > 32 ? 32 : k)];
    *row_bits = g.row_bits;
    *col_lw = g.col_lw;
    *rbits = g.rbits;
}

std::vector<int> ntt_pass_bits(int k, int form)
{
    // One in-CTA pass up to 2^13 points; then column passes of at most 11
    // bits (balanced) and the row pass.
    std::vector<int> bits;
    if (k <= kInnerBits) {
        bits.push_back(k);
        return bits;
    }
    const int row = g_geom_forms[form == kFormDbl ? 1 : 0][k].row_bits, colmax = 11;
    int rest = k - row;
    const int ncol = (rest + colmax - 1) / colmax;
    for (int i = 0; i < ncol; i++) {
        const int b = rest / (ncol - i) + ((rest % (ncol - i)) ? 1 : 0);
        bits.push_back(b);
        rest -= b;
    }
    bits.push_back(row);
    return bits;
}

// Column tile width for a column pass of 2^lc rows: enough columns that a CTA
// holds >= 4096 points (every thread busy in every radix-8 round), at least 4
// (a 32-byte DRAM sector per row), at most 64.
static int col_width_log2(int lc)
{
    int lw = 12 - lc;
    if (lw < 2) lw = 2;
    if (lw > 6) lw = 6;
    return lw;
}

// Compile-time kernel variants (chosen by measurement; see the profiles):
// PIC_NTT_PREFETCH loads a radix group's twiddles before its butterflies,
// PIC_NTT_SWIZZLE XOR-swizzles the row kernel's shared-memory layout.
#ifndef PIC_NTT_PREFETCH
#define PIC_NTT_PREFETCH 0
#endif
#ifndef PIC_NTT_SWIZZLE
#define PIC_NTT_SWIZZLE 1
#endif

#ifndef PIC_NTT_QP1
#define PIC_NTT_QP1 1
#endif
#ifndef PIC_NTT_DIT4
#define PIC_NTT_DIT4 1
#endif

// ---------------------------------------------------------------------------
// Butterflies.  Strict: operands and results in [0, p).  Lazy (Harvey 2014,
// primes below 2^61 so 8p < 2^64): forward operands and results in [0, 4p);
// inverse operands and results in [0, 8p) (PIC_NTT_DIT4: only the even input
// is brought back below 4p, one correction per butterfly).  The Shoup product
// is left without its final correction, for any 64-bit input.

// q * p mod 2^64.  Lazy primes have the form c * 2^32 + 1, so
// q p = q + ((q mod 2^32) c) 2^32 (mod 2^64): one 32-bit multiply-add.
__device__ __forceinline__ uint64_t mul_p_lo(uint64_t q, uint64_t p)
{
#if PIC_NTT_QP1
    const uint32_t c = (uint32_t)(p >> 32);
    return q + ((uint64_t)((uint32_t)q * c) << 32);
#else
    return q * p;
#endif
}

// x * w mod p in [0, 2p) (lazy primes), x < 2^64.
__device__ __forceinline__ uint64_t shoup_lazy(uint64_t x, uint64_t w, uint64_t ws, uint64_t p)
{
    return x * w - mul_p_lo(mulhi64(x, ws), p);
}

template <bool LAZY>
__device__ __forceinline__ void bfly_dif(uint64_t& a, uint64_t& b, uint64_t w, uint64_t ws, uint64_t p)
{
    if (LAZY) {
        const uint64_t p4 = 4 * p;
        uint64_t x = a + b;
        x = x >= p4 ? x - p4 : x;
        b = shoup_lazy(a + p4 - b, w, ws, p);
        a = x;
    } else {
        const uint64_t x = a, y = b;
        a = add_mod(x, y, p);
        b = shoup_mul(sub_mod(x, y, p), w, ws, p);
    }
}

// Butterfly with a unit twiddle (the h = 1 level): no multiplication.
template <bool LAZY>
__device__ __forceinline__ void bfly_unit(uint64_t& a, uint64_t& b, uint64_t p)
{
    if (LAZY) {
        const uint64_t p4 = 4 * p;
        uint64_t x = a + b;
        x = x >= p4 ? x - p4 : x;
        uint64_t y = a + p4 - b;
        y = y >= p4 ? y - p4 : y;
        a = x;
        b = y;
    } else {
        const uint64_t x = a, y = b;
        a = add_mod(x, y, p);
        b = sub_mod(x, y, p);
    }
}

// Inverse-direction unit butterfly: lazy operands in [0, 8p).
template <bool LAZY>
__device__ __forceinline__ void bfly_unit_dit(uint64_t& a, uint64_t& b, uint64_t p)
{
    if (LAZY) {
        const uint64_t p4 = 4 * p;
        const uint64_t x = a >= p4 ? a - p4 : a;
        const uint64_t y = b >= p4 ? b - p4 : b;
#if PIC_NTT_DIT4
        a = x + y;
        b = x + p4 - y;
#else
        a = x;
        b = y;
        bfly_unit<LAZY>(a, b, p);
#endif
        return;
    }
    bfly_unit<LAZY>(a, b, p);
}

template <bool LAZY>
__device__ __forceinline__ void bfly_dit(uint64_t& a, uint64_t& b, uint64_t w, uint64_t ws, uint64_t p)
{
    if (LAZY) {
        const uint64_t p4 = 4 * p;
        const uint64_t u = shoup_lazy(b, w, ws, p);
        const uint64_t x = a >= p4 ? a - p4 : a;
#if PIC_NTT_DIT4
        a = x + u;
        b = x + p4 - u;
#else
        uint64_t s = x + u;
        s = s >= p4 ? s - p4 : s;
        uint64_t d = x + p4 - u;
        d = d >= p4 ? d - p4 : d;
        a = s;
        b = d;
#endif
    } else {
        const uint64_t x = a, y = shoup_mul(b, w, ws, p);
        a = add_mod(x, y, p);
        b = sub_mod(x, y, p);
    }
}

// One group of 2^B elements at positions base + j + m * 2^lst of a sub-block
// of size 2^(lst + B); performs the B butterfly levels of that sub-block.  All
// 2^B - 1 twiddle pairs of the group are loaded before the first butterfly so
// their latencies overlap.
template <int B, bool INV, bool LAZY>
__device__ __forceinline__ void group_levels(uint64_t (&x)[1 << B], int j, int lst, uint64_t p, int IB,
                                             const uint64_t* __restrict__ tw)
{
    constexpr int NT = (1 << B) - 1;
    ulonglong2 w[NT];
    const bool unit_last = lst == 0;  // the h = 1 level has every twiddle equal to 1
#if PIC_NTT_PREFETCH
#pragma unroll
    for (int l = 0; l < B; l++) {
        const int hm = 1 << (B - 1 - l);
        const int off = (1 << B) - (1 << (B - l));
        if (l == B - 1 && unit_last) continue;
        const int shift = IB - (B - l) - lst;  // root of order 2h = 2^(B-l+lst)
#pragma unroll
        for (int u = 0; u < hm; u++)
            w[off + u] = __ldg(reinterpret_cast<const ulonglong2*>(tw) + ((j + (u << lst)) << shift));
    }
#define PIC_TW(l, u) w[(1 << B) - (1 << (B - (l))) + (u)]
#else
#define PIC_TW(l, u) \
    __ldg(reinterpret_cast<const ulonglong2*>(tw) + ((j + ((u) << lst)) << (IB - (B - (l)) - lst)))
#endif
    if (!INV) {
#pragma unroll
        for (int l = 0; l < B; l++) {
            const int hm = 1 << (B - 1 - l);
            if (l == B - 1 && unit_last) {
#pragma unroll
                for (int m = 0; m < (1 << B); m += 2) bfly_unit<LAZY>(x[m], x[m + 1], p);
                continue;
            }
#pragma unroll
            for (int m = 0; m < (1 << B); m++) {
                if (m & hm) continue;
                const ulonglong2 t = PIC_TW(l, m & (hm - 1));
                bfly_dif<LAZY>(x[m], x[m + hm], t.x, t.y, p);
            }
        }
    } else {
#pragma unroll
        for (int l = B - 1; l >= 0; l--) {
            const int hm = 1 << (B - 1 - l);
            if (l == B - 1 && unit_last) {
#pragma unroll
                for (int m = 0; m < (1 << B); m += 2) bfly_unit_dit<LAZY>(x[m], x[m + 1], p);
                continue;
            }
#pragma unroll
            for (int m = 0; m < (1 << B); m++) {
                if (m & hm) continue;
                const ulonglong2 t = PIC_TW(l, m & (hm - 1));
                bfly_dit<LAZY>(x[m], x[m + hm], t.x, t.y, p);
            }
        }
    }
#undef PIC_TW
    (void)w;
}

// Row layout swizzle: XOR bits 4..7 of an element's index into bits 0..3, a
// bijection on every row that spreads the small-stride rounds over all
// shared-memory banks.
__device__ __forceinline__ int swz(int e)
{
#if PIC_NTT_SWIZZLE
    return e ^ ((e >> 4) & 15);
#else
    return e;
#endif
}

template <int B, bool INV, bool LAZY, bool SWZ>
__device__ __forceinline__ void run_group(uint64_t* __restrict__ ptr, int base, int j, int lst, int les,
                                          uint64_t p, int IB, const uint64_t* tw)
{
    uint64_t x[1 << B];
#pragma unroll
    for (int m = 0; m < (1 << B); m++) {
        const int e = base + (m << lst);
        x[m] = ptr[SWZ ? swz(e) : (e << les)];
    }
    group_levels<B, INV, LAZY>(x, j, lst, p, IB, tw);
#pragma unroll
    for (int m = 0; m < (1 << B); m++) {
        const int e = base + (m << lst);
        ptr[SWZ ? swz(e) : (e << les)] = x[m];
    }
}

// 2^lnt transforms of size 2^logn in shared memory; element m of transform t
// lives at s[(t << lts) + (m << les)] (SWZ: s[(t << lts) + swz(m)], les = 0).
// tr_fast: consecutive threads walk transforms (column tiles), else elements
// (rows).
template <bool INV, bool LAZY, bool SWZ, int rb>
__device__ void cta_ntt(uint64_t* s, int logn, int lnt, int les, int lts, bool tr_fast, uint64_t p, int IB,
                        const uint64_t* tw)
{
    const int nfull = logn / rb, rem = logn % rb;
    const int nr = nfull + (rem ? 1 : 0);
    for (int ri = 0; ri < nr; ri++) {
        const int r = INV ? (nr - 1 - ri) : ri;
        const int b = (r < nfull) ? rb : rem;
        const int lB = logn - rb * r;  // log2 sub-block size
        const int lst = lB - b;       // log2 stride inside the group
        const int lgpt = logn - b;    // log2 groups per transform
        const int G = 1 << (lnt + lgpt);
        for (int g = threadIdx.x; g < G; g += blockDim.x) {
            int tr, gi;
            if (tr_fast) {
                tr = g & ((1 << lnt) - 1);
                gi = g >> lnt;
            } else {
                tr = g >> lgpt;
                gi = g & ((1 << lgpt) - 1);
            }
            const int j = gi & ((1 << lst) - 1);
            const int base = ((gi >> lst) << lB) + j;
            uint64_t* ptr = s + (tr << lts);
            if (rb >= 4 && b == 4) run_group<(rb >= 4 ? 4 : 1), INV, LAZY, SWZ>(ptr, base, j, lst, les, p, IB, tw);
            else if (b == 3) run_group<3, INV, LAZY, SWZ>(ptr, base, j, lst, les, p, IB, tw);
            else if (b == 2) run_group<2, INV, LAZY, SWZ>(ptr, base, j, lst, les, p, IB, tw);
            else run_group<1, INV, LAZY, SWZ>(ptr, base, j, lst, les, p, IB, tw);
        }
        __syncthreads();
    }
}

// Constant-index selection keeps the prime's fields in registers (a dynamic
// index into the kernel's parameter array would spill the array to local memory).
__device__ __forceinline__ PrimeDev pick_prime(const NttBatch& B, int tr)
{
    return tr < B.per_prime ? B.prime[0] : (tr < 2 * B.per_prime ? B.prime[1] : B.prime[2]);
}

// Root of unity w_(2^lM)^e in Montgomery form from the two-level tables.
template <bool INV>
__device__ __forceinline__ uint64_t outer_root(const PrimeDev& P, uint64_t e, int lM)
{
    const uint64_t E = e << (P.K - lM);
    const uint64_t lo = E & ((1ull << P.S) - 1), hi = E >> P.S;
    const uint64_t* tl = INV ? P.olo_inv : P.olo_fwd;
    const uint64_t* th = INV ? P.ohi_inv : P.ohi_fwd;
    return mont_mul(__ldg(th + hi), __ldg(tl + lo), P.p, P.pinv_neg);
}

// Contiguous row pass: rows of 2^lr elements; 2^lrpc rows per CTA.
template <bool INV, bool LAZY, int RB>
__global__ void __launch_bounds__(512) ntt_rows_kernel(NttBatch B, int k, int lr, int lrpc)
{
    extern __shared__ uint64_t smem[];
    const int lrow = k - lr;  // log2 rows per transform
    const size_t row0 = (size_t)blockIdx.x << lrpc;
    const int tr0 = (int)(row0 >> lrow);
    const PrimeDev P = pick_prime(B, tr0);
    const int tot = 1 << (lrpc + lr);
    const size_t rmask = ((size_t)1 << lrow) - 1;
    const int emask = (1 << lr) - 1;
    for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
        const size_t row = row0 + (idx >> lr);
        smem[(idx & ~emask) + swz(idx & emask)] =
            B.data[(row >> lrow) * B.stride + ((row & rmask) << lr) + (idx & emask)];
    }
    __syncthreads();
    cta_ntt<INV, LAZY, true, RB>(smem, lr, lrpc, 0, lr, false, P.p, P.IB, INV ? P.inner_inv : P.inner_fwd);
    for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
        const size_t row = row0 + (idx >> lr);
        B.data[(row >> lrow) * B.stride + ((row & rmask) << lr) + (idx & emask)] =
            smem[(idx & ~emask) + swz(idx & emask)];
    }
}

// Strided column pass.  The transform is a sequence of 2^lpre outer blocks of
// 2^(k-lpre) elements; each outer block is an N1 x M tile (N1 = 2^lc rows,
// M = 2^(k-lpre-lc) columns, row-major).  A CTA owns 2^lw columns of one tile.
template <bool INV, bool LAZY, int RB>
__global__ void __launch_bounds__(256) ntt_cols_kernel(NttBatch B, int k, int lpre, int lc, int lw)
{
    extern __shared__ uint64_t smem[];
    const int lM = k - lpre - lc;
    const int ltiles = lM - lw;  // log2 tiles per outer block
    const size_t cta = blockIdx.x;
    const int tr = (int)(cta >> (ltiles + lpre));
    const size_t rem = cta & (((size_t)1 << (ltiles + lpre)) - 1);
    const size_t ob = rem >> ltiles;
    const size_t c0 = (rem & (((size_t)1 << ltiles) - 1)) << lw;
    const PrimeDev P = pick_prime(B, tr);
    uint64_t* base = B.data + (size_t)tr * B.stride + (ob << (k - lpre)) + c0;
    const int tot = 1 << (lc + lw);
    const int lblock = k - lpre;  // twiddle root order 2^lblock
    const int wmask = (1 << lw) - 1;
    for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
        const int m = idx >> lw, w = idx & wmask;
        uint64_t v = base[((size_t)m << lM) + w];
        if (INV) {
            const uint64_t k1 = __brev((unsigned)m) >> (32 - lc);
            v = mont_mul(v, outer_root<true>(P, (c0 + w) * k1, lblock), P.p, P.pinv_neg);
        }
        smem[idx] = v;
    }
    __syncthreads();
    cta_ntt<INV, LAZY, false, RB>(smem, lc, lw, lw, 0, true, P.p, P.IB, INV ? P.inner_inv : P.inner_fwd);
    for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
        const int m = idx >> lw, w = idx & wmask;
        uint64_t v = smem[idx];
        if (!INV) {
            const uint64_t k1 = __brev((unsigned)m) >> (32 - lc);
            v = mont_mul(v, outer_root<false>(P, (c0 + w) * k1, lblock), P.p, P.pinv_neg);
        }
        base[((size_t)m << lM) + w] = v;
    }
}

// ---------------------------------------------------------------------------
// Fast path for the lazy primes (c * 2^32 + 1 < 2^62, inner tables of order
// 2^13): every geometry parameter of a pass is a compile-time constant, so the
// group, stride and twiddle index arithmetic folds away, and the Shoup product
// is written with explicit 32-bit multiply-adds and carries.

#ifndef PIC_NTT_FAST
#define PIC_NTT_FAST 1
#endif

struct LazyPrime {
    uint64_t p, p4;
    uint32_t c;  // p = c * 2^32 + 1
};

__device__ __forceinline__ LazyPrime lazy_prime(const PrimeDev& P)
{
    LazyPrime L;
    L.p = P.p;
    L.p4 = 4 * P.p;
    L.c = (uint32_t)(P.p >> 32);
    return L;
}

// Piece j of batch item tr from the item's child slot (SplitSrc), reduced to
// [0, 4p) (a 64-bit piece is below 9p for the lazy primes).
struct SrcRow {
    const uint32_t* x;
    uint32_t n;
};

__device__ __forceinline__ SrcRow src_row(const NttBatch& B, int tr)
{
    const size_t c = B.src.c0 + (size_t)(tr % B.per_prime);
    SrcRow r;
    r.x = B.src.words + c * (size_t)B.src.cap;
    r.n = B.src.len[c];
    return r;
}

__device__ __forceinline__ uint64_t src_piece_raw(const NttBatch& B, const SrcRow& r, size_t j)
{
    const size_t wi = 2 * (B.src.first + j);
    uint64_t v = 0;
    if (wi < r.n) {
        v = __ldg(r.x + wi);
        if (wi + 1 < r.n) v |= (uint64_t)__ldg(r.x + wi + 1) << 32;
    }
    return v;
}

__device__ __forceinline__ uint64_t src_piece(const NttBatch& B, const SrcRow& r, size_t j, uint64_t p4)
{
    return piece_to_lazy(src_piece_raw(B, r, j), p4);
}

// Forward (DIF): operands and results in [0, 4p).
__device__ __forceinline__ void fbfly_dif(uint64_t& a, uint64_t& b, const ulonglong2 t, const LazyPrime& L)
{
    uint64_t x = a + b;
    x = x >= L.p4 ? x - L.p4 : x;
    b = shoup_approx32(a + L.p4 - b, t.x, t.y, L.c);
    a = x;
}

__device__ __forceinline__ void fbfly_unit_dif(uint64_t& a, uint64_t& b, const LazyPrime& L)
{
    uint64_t x = a + b;
    x = x >= L.p4 ? x - L.p4 : x;
    uint64_t y = a + L.p4 - b;
    y = y >= L.p4 ? y - L.p4 : y;
    a = x;
    b = y;
}

// Inverse (DIT): operands and results in [0, 8p).
__device__ __forceinline__ void fbfly_dit(uint64_t& a, uint64_t& b, const ulonglong2 t, const LazyPrime& L)
{
    const uint64_t u = shoup_approx32(b, t.x, t.y, L.c);
    const uint64_t x = a >= L.p4 ? a - L.p4 : a;
    a = x + u;
    b = x + L.p4 - u;
}

__device__ __forceinline__ void fbfly_unit_dit(uint64_t& a, uint64_t& b, const LazyPrime& L)
{
    const uint64_t x = a >= L.p4 ? a - L.p4 : a;
    const uint64_t y = b >= L.p4 ? b - L.p4 : b;
    a = x + y;
    b = x + L.p4 - y;
}

// Arithmetic of the fast passes.  ArithInt: lazy Shoup butterflies on 64-bit
// residues (lazy primes).  ArithDbl: FP64 butterflies (FP64 primes, values
// stored as the bits of doubles; twiddles w form their companion per use,
// so a product lands below p).  `LAST` marks the last level of a register
// round: the FP64 forward butterflies reduce their sums there, so every
// round starts and ends with |x| <= p; inside a round of B levels the values
// stay below 2^B p (16 p for radix-16, under 2^51 for primes below 2^47).
// FP64 inverse butterflies add at most p per level and never reduce: a pass
// of L levels over inputs below X ends below 2 X + (L - 1) p (15 p for a
// 13-level row pass over the merges' T1 +- T2, below 1.5 p).
struct ArithInt {
    using T = uint64_t;
    using Tw = ulonglong2;  // twiddle table entry: Shoup pair (w, w')
    using Ctx = LazyPrime;
    static __device__ __forceinline__ Ctx ctx(const PrimeDev& P) { return lazy_prime(P); }
    static __device__ __forceinline__ T ld(uint64_t v) { return v; }
    static __device__ __forceinline__ uint64_t st(T v) { return v; }
    template <bool LAST>
    static __device__ __forceinline__ void dif(T& a, T& b, const ulonglong2 t, const Ctx& L) { fbfly_dif(a, b, t, L); }
    template <bool LAST>
    static __device__ __forceinline__ void dif_unit(T& a, T& b, const Ctx& L) { fbfly_unit_dif(a, b, L); }
    static __device__ __forceinline__ void dit(T& a, T& b, const ulonglong2 t, const Ctx& L) { fbfly_dit(a, b, t, L); }
    static __device__ __forceinline__ void dit_unit(T& a, T& b, const Ctx& L) { fbfly_unit_dit(a, b, L); }
    // v * w (pass twiddle) into [0, 4p) from any 64-bit v
    static __device__ __forceinline__ T twiddle(T v, const ulonglong2 t, const Ctx& L)
    {
        return shoup_approx32(v, t.x, t.y, L.c);
    }
    // piece j of the item's child words, as a residue
    static __device__ __forceinline__ T piece(const NttBatch& B, const SrcRow& r, size_t j, const Ctx& L)
    {
        return src_piece(B, r, j, L.p4);
    }
};

struct ArithDbl {
    using T = double;
    using Tw = double;  // twiddle table entry: w; the companion is formed per use (dmul_w)
    struct Ctx {
        double p, pinv;
    };
    static __device__ __forceinline__ Ctx ctx(const PrimeDev& P) { return Ctx{P.pd, P.pinv}; }
    static __device__ __forceinline__ T ld(uint64_t v) { return dbits(v); }
    static __device__ __forceinline__ uint64_t st(T v) { return dstore(v); }
    template <bool LAST>
    static __device__ __forceinline__ void dif(T& a, T& b, const Tw t, const Ctx& L)
    {
        const double s = __dadd_rn(a, b), d = __dadd_rn(a, -b);
        b = dmul_w(d, t, L.p, L.pinv);
        a = LAST ? dreduce(s, L.p, L.pinv) : s;
    }
    template <bool LAST>
    static __device__ __forceinline__ void dif_unit(T& a, T& b, const Ctx& L)
    {
        const double s = __dadd_rn(a, b), d = __dadd_rn(a, -b);
        a = LAST ? dreduce(s, L.p, L.pinv) : s;
        b = LAST ? dreduce(d, L.p, L.pinv) : d;
    }
    static __device__ __forceinline__ void dit(T& a, T& b, const Tw t, const Ctx& L)
    {
        const double u = dmul_w(b, t, L.p, L.pinv);
        b = __dadd_rn(a, -u);
        a = __dadd_rn(a, u);
    }
    static __device__ __forceinline__ void dit_unit(T& a, T& b, const Ctx&)
    {
        const double s = __dadd_rn(a, b);
        b = __dadd_rn(a, -b);
        a = s;
    }
    static __device__ __forceinline__ T twiddle(T v, const Tw t, const Ctx& L) { return dmul_w(v, t, L.p, L.pinv); }
    static __device__ __forceinline__ T piece(const NttBatch& B, const SrcRow& r, size_t j, const Ctx& L)
    {
        return dpiece56(src_piece56_raw(r.x, r.n, B.src.first + j), L.p, L.pinv);
    }
};

// The B levels of one group (elements base + j + m 2^LST, m < 2^B) with the
// per-level inner tables: the twiddle of butterfly u at group level l is
// root_(2^(B-l+LST))^(j + u 2^LST), pair 2^(B-l+LST-1) - 1 + j + u 2^LST, so
// lanes with consecutive j read consecutive pairs.
template <int B, bool INV, int LST, class A>
__device__ __forceinline__ void group_fast(typename A::T (&x)[1 << B], int j, const typename A::Ctx& L,
                                           const typename A::Tw* __restrict__ tw)
{
    static_assert(B + LST <= 13, "sub-block larger than the inner table");
    if (!INV) {
#pragma unroll
        for (int l = 0; l < B; l++) {
            const int hm = 1 << (B - 1 - l);
            if (l == B - 1 && LST == 0) {
#pragma unroll
                for (int m = 0; m < (1 << B); m += 2) A::template dif_unit<true>(x[m], x[m + 1], L);
                continue;
            }
#pragma unroll
            for (int m = 0; m < (1 << B); m++) {
                if (m & hm) continue;
                const int u = m & (hm - 1);
                const typename A::Tw t = __ldg(tw + ((1 << (B - l + LST - 1)) - 1) + j + (u << LST));
                if (l == B - 1) A::template dif<true>(x[m], x[m + hm], t, L);
                else A::template dif<false>(x[m], x[m + hm], t, L);
            }
        }
    } else {
#pragma unroll
        for (int l = B - 1; l >= 0; l--) {
            const int hm = 1 << (B - 1 - l);
            if (l == B - 1 && LST == 0) {
#pragma unroll
                for (int m = 0; m < (1 << B); m += 2) A::dit_unit(x[m], x[m + 1], L);
                continue;
            }
#pragma unroll
            for (int m = 0; m < (1 << B); m++) {
                if (m & hm) continue;
                const int u = m & (hm - 1);
                A::dit(x[m], x[m + hm], __ldg(tw + ((1 << (B - l + LST - 1)) - 1) + j + (u << LST)), L);
            }
        }
    }
}

// Radix-2^RB rounds of a 2^LOGN transform (plus one smaller round when RB
// does not divide LOGN, at the smallest stride); forward rounds run from the
// largest stride down, inverse rounds the other way.
template <int LOGN, int RB = 3>
struct RoundPlan {
    static constexpr int NF = LOGN / RB, REM = LOGN % RB, NR = NF + (REM ? 1 : 0);
    template <int RR>
    struct At {
        static constexpr int B = RR < NF ? RB : REM;
        static constexpr int LB = LOGN - RB * RR;  // log2 sub-block size
        static constexpr int LST = LB - B;         // log2 stride inside a group
    };
};

// Row layout: transform t of the CTA at s + (t << LR), element e at swz(e).
// With several transforms per CTA (LRPC > 0, single-pass lengths), each
// group takes the prime of its own transform: a CTA may straddle primes.
// The first round reads its groups straight from global memory through
// in(t, e, ctx) (forward: the largest stride, consecutive lanes read
// consecutive points; inverse: a run of 2^B points per lane, through L1);
// with OUT_DIRECT the last round (inverse: the largest stride again) writes
// through out(t, e, v).  The rounds between exchange through shared memory.
template <bool INV, int LR, int LRPC, int NT, int RB, int R, bool OUT_DIRECT, class A, class In, class Out>
__device__ __forceinline__ void rows_fast_round(uint64_t* __restrict__ s, const NttBatch& Bt, size_t row0,
                                                const typename A::Ctx& L0, const typename A::Tw* __restrict__ tw0,
                                                const In& in, const Out& out)
{
    using Plan = RoundPlan<LR, RB>;
    constexpr int RR = INV ? Plan::NR - 1 - R : R;
    using At = typename Plan::template At<RR>;
    constexpr int B = At::B, LB = At::LB, LST = At::LST;
    constexpr int LG = LR - B;  // log2 groups per transform
    constexpr int G = 1 << (LRPC + LG);
    constexpr bool LAST = R + 1 == Plan::NR;
    static_assert(G % NT == 0, "groups must split evenly over the threads");
#pragma unroll
    for (int q = 0; q < G / NT; q++) {
        const int g = threadIdx.x + q * NT;
        const int t = g >> LG, gi = g & ((1 << LG) - 1);
        const int j = gi & ((1 << LST) - 1);
        const int base = ((gi >> LST) << LB) + j;
        uint64_t* ptr = s + (t << LR);
        typename A::Ctx L = L0;
        const typename A::Tw* tw = tw0;
        if (LRPC > 0 && row0 + t < (size_t)Bt.count) {  // rows past the batch keep the CTA's prime
            const PrimeDev Pt = pick_prime(Bt, (int)(row0 + t));
            L = A::ctx(Pt);
            tw = reinterpret_cast<const typename A::Tw*>(INV ? Pt.lvl_inv : Pt.lvl_fwd);
        }
        typename A::T x[1 << B];
#pragma unroll
        for (int m = 0; m < (1 << B); m++) {
            const int e = base + (m << LST);
            if constexpr (R == 0) x[m] = in(t, e, L);
            else x[m] = A::ld(ptr[swz(e)]);
        }
        group_fast<B, INV, LST, A>(x, j, L, tw);
#pragma unroll
        for (int m = 0; m < (1 << B); m++) {
            const int e = base + (m << LST);
            if constexpr (LAST && OUT_DIRECT) out(t, e, x[m]);
            else ptr[swz(e)] = A::st(x[m]);
        }
    }
    if constexpr (!(LAST && OUT_DIRECT)) __syncthreads();
    if constexpr (!LAST)
        rows_fast_round<INV, LR, LRPC, NT, RB, R + 1, OUT_DIRECT, A>(s, Bt, row0, L0, tw0, in, out);
}

// One thread per group of a full round: 2^(LR + LRPC - RB) threads, at most
// 512.  Radix-16 groups hold 16 residues per thread, so that form runs one
// CTA of up to 512 threads per SM with room for 128 registers a thread.
template <int LR, int LRPC, int RB = 3>
struct RowsFastShape {
    static constexpr int TOT = 1 << (LR + LRPC);
    static constexpr int NT = (TOT >> RB) > 512 ? 512 : ((TOT >> RB) < 32 ? 32 : (TOT >> RB));
    static constexpr int MINB = RB == 3 ? 1024 / NT : 1;
};

// Contiguous row pass: 2^LRPC rows of 2^LR points per CTA.  LRPC > 0 only
// for single-pass lengths (k = LR, one row per transform); the last CTA may
// hold fewer than 2^LRPC transforms.  Forward passes stage their output
// through shared memory (their last round has the smallest stride); inverse
// passes write it directly.
template <bool INV, int LR, int LRPC, int RB, class A>
__global__ void __launch_bounds__(RowsFastShape<LR, LRPC, RB>::NT, RowsFastShape<LR, LRPC, RB>::MINB)
    ntt_rows_fast_kernel(NttBatch B, int k)
{
    extern __shared__ uint64_t smem[];
    constexpr int TOT = RowsFastShape<LR, LRPC, RB>::TOT, NT = RowsFastShape<LR, LRPC, RB>::NT;
    constexpr int EMASK = (1 << LR) - 1;
    const int lrow = k - LR;  // log2 rows per transform
    const size_t rmask = ((size_t)1 << lrow) - 1;
    const size_t row0 = (size_t)blockIdx.x << LRPC;
    const size_t nrows = (size_t)B.count << lrow;
    const PrimeDev P = pick_prime(B, (int)(row0 >> lrow));
    const typename A::Ctx L = A::ctx(P);
    const bool from_src = !INV && B.src.words != nullptr;  // single-pass length: row == transform
    uint64_t* __restrict__ data = B.data;
    auto at = [&](int t, int e) {
        const size_t row = row0 + t;
        return (row >> lrow) * B.stride + ((row & rmask) << LR) + e;
    };
    auto in = [&](int t, int e, const typename A::Ctx& Lt) -> typename A::T {
        if (LRPC > 0 && row0 + t >= nrows) return A::ld(0);
        if (from_src) return A::piece(B, src_row(B, (int)(row0 + t)), e, Lt);
        return A::ld(data[at(t, e)]);
    };
    auto out = [&](int t, int e, typename A::T v) {
        if (LRPC == 0 || row0 + t < nrows) data[at(t, e)] = A::st(v);
    };
    rows_fast_round<INV, LR, LRPC, NT, RB, 0, INV, A>(
        smem, B, row0, L, reinterpret_cast<const typename A::Tw*>(INV ? P.lvl_inv : P.lvl_fwd), in, out);
    if constexpr (!INV) {
#pragma unroll
        for (int i = 0; i < TOT / NT; i++) {
            const int idx = threadIdx.x + i * NT;
            const size_t row = row0 + (idx >> LR);
            if (LRPC == 0 || row < nrows)
                data[(row >> lrow) * B.stride + ((row & rmask) << LR) + (idx & EMASK)] =
                    smem[(idx & ~EMASK) + swz(idx & EMASK)];
        }
    }
}

// Column tile: 2^LC rows x 2^LW columns, element (m, w) at s[(m << LW) + w];
// consecutive threads take consecutive columns.  The first round reads
// global memory through in(m, w) and the last writes it through
// out(m, w, v), both in runs of 2^LW consecutive points; the rounds between
// exchange through shared memory.
// PIC_COLS_TW_PREFETCH (default on): the last forward round loads its
// pass-table twiddles before its butterflies, so their latency overlaps the
// arithmetic (out(r, w, v, t) then applies them).
#ifndef PIC_COLS_TW_PREFETCH
#define PIC_COLS_TW_PREFETCH 1
#endif

template <bool INV, int LC, int LW, int RB, int R, class A, class In, class Out, class Pre>
__device__ __forceinline__ void cols_fast_round(uint64_t* __restrict__ s, const typename A::Ctx& L,
                                                const typename A::Tw* __restrict__ tw, const In& in, const Out& out,
                                                const Pre& pre)
{
    using Plan = RoundPlan<LC, RB>;
    constexpr int RR = INV ? Plan::NR - 1 - R : R;
    using At = typename Plan::template At<RR>;
    constexpr int B = At::B, LB = At::LB, LST = At::LST;
    constexpr int LG = LC - B;  // log2 groups per column
    constexpr int G = 1 << (LW + LG);
    constexpr int WMASK = (1 << LW) - 1;
    constexpr bool LAST = R + 1 == Plan::NR;
#pragma unroll
    for (int g = threadIdx.x; g < G; g += 256) {
        const int w = g & WMASK, gi = g >> LW;
        const int j = gi & ((1 << LST) - 1);
        const int base = ((gi >> LST) << LB) + j;
        typename A::T x[1 << B];
#pragma unroll
        for (int m = 0; m < (1 << B); m++) {
            const int r = base + (m << LST);
            if constexpr (R == 0) x[m] = in(r, w);
            else x[m] = A::ld(s[(r << LW) + w]);
        }
        constexpr bool PRE = LAST && !INV && PIC_COLS_TW_PREFETCH;
        typename A::Tw tp[PRE ? (1 << B) : 1];
        if constexpr (PRE) {
#pragma unroll
            for (int m = 0; m < (1 << B); m++) tp[m] = pre(base + (m << LST), w);
        }
        group_fast<B, INV, LST, A>(x, j, L, tw);
#pragma unroll
        for (int m = 0; m < (1 << B); m++) {
            const int r = base + (m << LST);
            if constexpr (PRE) out(r, w, x[m], &tp[m]);
            else if constexpr (LAST) out(r, w, x[m], nullptr);
            else s[(r << LW) + w] = A::st(x[m]);
        }
    }
    if constexpr (!LAST) {
        __syncthreads();
        cols_fast_round<INV, LC, LW, RB, R + 1, A>(s, L, tw, in, out, pre);
    }
}

// floor(x 2^64 / p) for x < p: q' = floor(x mu / 2^64) with mu = floor(2^128 /
// p) is q or q - 1 (x < 2^62), and the remainder x 2^64 - q' p < 2p decides.
__device__ __forceinline__ uint64_t shoup_companion_dev(uint64_t x, uint64_t p, uint64_t mu_hi, uint64_t mu_lo)
{
    const uint64_t q = x * mu_hi + __umul64hi(x, mu_lo);
    const uint64_t r = (uint64_t)0 - q * p;
    return r >= p ? q + 1 : q;
}

// Pass twiddle tables: for a column pass over blocks of 2^lblock points split
// 2^LC x M, entry m M + c = root_(2^lblock)^(+-c brev_LC(m)) as a Shoup pair
// (FP64 primes: the pair (w, fl(w / p)) of doubles), laid out like the data
// so the pass streams it with the same coalescing.
struct PassTw {
    const void* t[kMaxPrimesPerBatch];  // ulonglong2 Shoup pairs, or doubles (FP64 primes)
};

__global__ void pass_table_kernel(void* __restrict__ out_v, PrimeDev P, int inv, int lblock, int lc)
{
    const size_t n = (size_t)1 << lblock;
    const int lM = lblock - lc;
    const int esh = P.K - lblock;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < n; g += (size_t)gridDim.x * blockDim.x) {
        const uint64_t m = g >> lM, c = g & (((size_t)1 << lM) - 1);
        const uint64_t k1 = __brev((unsigned)m) >> (32 - lc);
        const uint64_t E = (c * k1) << esh;
        const uint64_t ehi = E >> P.S, elo = E & (((uint64_t)1 << P.S) - 1);
        if (P.fp64) {  // doubles w, |w| < p after dmul_w, brought into [0, p)
            const double* dlo = reinterpret_cast<const double*>(inv ? P.slo_inv : P.slo_fwd);
            const double* dhi = reinterpret_cast<const double*>(inv ? P.shi_inv : P.shi_fwd);
            double x = dmul_w(__ldg(dhi + ehi), __ldg(dlo + elo), P.pd, P.pinv);
            x = dcanon(x >= P.pd ? __dadd_rn(x, -P.pd) : x, P.pd);
            reinterpret_cast<double*>(out_v)[g] = x;
            continue;
        }
        const ulonglong2* slo = reinterpret_cast<const ulonglong2*>(inv ? P.slo_inv : P.slo_fwd);
        const ulonglong2* shi = reinterpret_cast<const ulonglong2*>(inv ? P.shi_inv : P.shi_fwd);
        ulonglong2* out = reinterpret_cast<ulonglong2*>(out_v);
        const ulonglong2 h = __ldg(shi + ehi), l = __ldg(slo + elo);
        const LazyPrime L = lazy_prime(P);
        uint64_t x = shoup_lazy32(h.x, l.x, l.y, L.c);
        x = x >= L.p ? x - L.p : x;
        out[g] = make_ulonglong2(x, shoup_companion_dev(x, L.p, P.mu_hi, P.mu_lo));
    }
}

// Strided column pass (same tiling as ntt_cols_kernel).  The inter-pass
// twiddle root_(2^lblock)^((c0 + w) k1) is applied as one product with the
// pass table, or as two with the two-level outer tables: forward after the
// column DIF, inverse before the column DIT.  The tile is read by the first
// register round and written by the last, without staging.
// RB 4: radix-16 rounds, 16 residues per thread, two CTAs per SM.
// Resident CTAs per SM the column kernels are compiled for (the register
// budget): radix-16 two; radix-8 integer four forward, three inverse; FP64
// PIC_DBL_COLS_MINB.
#ifndef PIC_DBL_COLS_MINB
#define PIC_DBL_COLS_MINB 4
#endif
template <class A, int RB, bool INV>
struct ColsMinBlocks {
    static constexpr int value = RB == 4 ? 2 : (std::is_same<A, ArithDbl>::value ? PIC_DBL_COLS_MINB : (INV ? 3 : 4));
};

template <bool INV, int LC, int LW, int RB, class A>
__global__ void __launch_bounds__(256, ColsMinBlocks<A, RB, INV>::value)
    ntt_cols_fast_kernel(NttBatch B, int k, int lpre, PassTw pt)
{
    extern __shared__ uint64_t smem[];
    const int lM = k - lpre - LC;
    const int ltiles = lM - LW;
    const size_t cta = blockIdx.x;
    const int tr = (int)(cta >> (ltiles + lpre));
    const size_t rem = cta & (((size_t)1 << (ltiles + lpre)) - 1);
    const size_t ob = rem >> ltiles;
    const uint32_t c0 = (uint32_t)((rem & (((size_t)1 << ltiles) - 1)) << LW);
    const PrimeDev P = pick_prime(B, tr);
    const typename A::Ctx L = A::ctx(P);
    uint64_t* base = B.data + (size_t)tr * B.stride + (ob << (k - lpre)) + c0;
    const int esh = P.K - (k - lpre);  // exponents of a root of order 2^(k - lpre), scaled to order 2^K
    const int S = P.S;
    const uint64_t smask = ((uint64_t)1 << S) - 1;
    using Tw = typename A::Tw;
    const Tw* __restrict__ slo = reinterpret_cast<const Tw*>(INV ? P.slo_inv : P.slo_fwd);
    const Tw* __restrict__ shi = reinterpret_cast<const Tw*>(INV ? P.shi_inv : P.shi_fwd);
    const Tw* __restrict__ T =
        static_cast<const Tw*>(tr < B.per_prime ? pt.t[0] : (tr < 2 * B.per_prime ? pt.t[1] : pt.t[2]));
    auto twiddle = [&](typename A::T v, int m, int w) {
        if (T != nullptr)  // the pass table: one product, streamed like the data
            return A::twiddle(v, __ldg(T + ((size_t)m << lM) + c0 + w), L);
        const uint64_t k1 = __brev((unsigned)m) >> (32 - LC);
        const uint64_t E = ((uint64_t)(c0 + w) * k1) << esh;
        const Tw h = __ldg(shi + (E >> S)), l = __ldg(slo + (E & smask));
        return A::twiddle(A::twiddle(v, h, L), l, L);
    };
    // first forward column pass (lpre == 0) with a split source: point
    // m M + c0 + w comes from the child slot
    const bool from_src = !INV && B.src.words != nullptr;
    const SrcRow sr = from_src ? src_row(B, tr) : SrcRow{nullptr, 0};
    auto in = [&](int m, int w) -> typename A::T {
        if (from_src) return A::piece(B, sr, ((size_t)m << lM) + c0 + w, L);
        const typename A::T v = A::ld(base[((size_t)m << lM) + w]);
        return INV ? twiddle(v, m, w) : v;
    };
    // pre(m, w): the pass-table pair of point (m, w) (zero without a table);
    // out applies a preloaded pair when it gets one
    auto pre = [&](int m, int w) -> Tw { return T != nullptr ? __ldg(T + ((size_t)m << lM) + c0 + w) : Tw{}; };
    auto out = [&](int m, int w, typename A::T v, const Tw* t) {
        if (!INV) v = (t != nullptr && T != nullptr) ? A::twiddle(v, *t, L) : twiddle(v, m, w);
        base[((size_t)m << lM) + w] = A::st(v);
    };
    cols_fast_round<INV, LC, LW, RB, 0, A>(smem, L,
                                           reinterpret_cast<const Tw*>(INV ? P.lvl_inv : P.lvl_fwd), in, out, pre);
}

// ---- column passes fed by TMA bulk copies ------------------------------------
// A persistent CTA walks the tiles t = blockIdx.x, blockIdx.x + gridDim.x, ...
// Each row of a tile (2^LW consecutive points, and the matching 2^LW pass-table
// pairs) is one contiguous, 16-byte-aligned run, so warp 0 fetches a tile with
// 2^LC bulk copies (plain cp.async.bulk into the CTA's own shared memory) that complete on an
// mbarrier; two buffers let the copies of tile i + 1 land while tile i is
// computed.  Every wait is bounded: a wait that outlasts ~1 s of SM clocks
// sets g_ntt_bulk_error, drains the other buffer's copy (also bounded) and
// ends the CTA; the host turns the flag into PIC_ERR_TIMEOUT.

__device__ int g_ntt_bulk_error;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase with the given parity; false after ~2^31 SM clocks.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity)
{
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > (1ll << 31)) return false;
    return true;
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

struct BulkTile {
    int tr;
    uint64_t* base;        // the tile's first point (row 0, column c0)
    const double* T;       // its pass-table rows (FP64 twiddles w; null: two-level tables)
    uint32_t c0;
};

__device__ __forceinline__ BulkTile bulk_tile(const NttBatch& B, const PassTw& pt, int k, int lpre, int lM, int LW,
                                              size_t t)
{
    const int ltiles = lM - LW;
    BulkTile r;
    r.tr = (int)(t >> (ltiles + lpre));
    const size_t rem = t & (((size_t)1 << (ltiles + lpre)) - 1);
    const size_t ob = rem >> ltiles;
    r.c0 = (uint32_t)((rem & (((size_t)1 << ltiles) - 1)) << LW);
    r.base = B.data + (size_t)r.tr * B.stride + (ob << (k - lpre)) + r.c0;
    r.T = static_cast<const double*>(r.tr < B.per_prime ? pt.t[0] : (r.tr < 2 * B.per_prime ? pt.t[1] : pt.t[2]));
    return r;
}

// Warp 0 fetches tile t into (d, tb) completing on bar.
template <int LC, int LW>
__device__ __forceinline__ void bulk_fetch(const BulkTile& tl, int lM, uint64_t* d, double* tb, uint64_t* bar)
{
    const int lane = threadIdx.x & 31;
    const uint32_t bytes = (uint32_t)((8u + (tl.T != nullptr ? 8u : 0u)) << (LC + LW));
    if (lane == 0) mbar_expect_tx(bar, bytes);
    __syncwarp();
    for (int m = lane; m < (1 << LC); m += 32) {
        bulk_load(d + (m << LW), tl.base + ((size_t)m << lM), 8u << LW, bar);
        if (tl.T != nullptr) bulk_load(tb + (m << LW), tl.T + ((size_t)m << lM) + tl.c0, 8u << LW, bar);
    }
}

template <int LC, int LW, bool TAB>
struct BulkShape {
    static constexpr int TOT = 1 << (LC + LW);
    static constexpr size_t DATA = sizeof(uint64_t) * TOT;
    static constexpr size_t TABB = TAB ? sizeof(double) * TOT : 0;
    static constexpr size_t SMEM = 2 * (DATA + TABB) + 64;  // two buffers and the barriers
};

template <bool INV, int LC, int LW, int RB, bool TAB, class A>
__global__ void __launch_bounds__(256, 2) ntt_cols_bulk_kernel(NttBatch B, int k, int lpre, PassTw pt, size_t ntiles)
{
    using Sh = BulkShape<LC, LW, TAB>;
    extern __shared__ __align__(128) uint64_t bsm[];
    uint64_t* dbuf[2] = {bsm, bsm + Sh::TOT};
    double* tbuf[2] = {reinterpret_cast<double*>(bsm + 2 * Sh::TOT), reinterpret_cast<double*>(bsm + 3 * Sh::TOT)};
    uint64_t* bars = reinterpret_cast<uint64_t*>(reinterpret_cast<char*>(bsm) + 2 * (Sh::DATA + Sh::TABB));
    const int lM = k - lpre - LC;
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        fence_async_smem();
    }
    __syncthreads();
    const size_t t0 = blockIdx.x, step = gridDim.x;
    if (threadIdx.x < 32) {
        if (t0 < ntiles) bulk_fetch<LC, LW>(bulk_tile(B, pt, k, lpre, lM, LW, t0), lM, dbuf[0], tbuf[0], &bars[0]);
        if (t0 + step < ntiles)
            bulk_fetch<LC, LW>(bulk_tile(B, pt, k, lpre, lM, LW, t0 + step), lM, dbuf[1], tbuf[1], &bars[1]);
    }
    size_t it = 0;
    for (size_t t = t0; t < ntiles; t += step, it++) {
        const int b = (int)(it & 1);
        const bool ok = mbar_wait_bounded(&bars[b], (uint32_t)((it >> 1) & 1));
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) {
                atomicExch(&g_ntt_bulk_error, 1);
                if (t + step < ntiles) mbar_wait_bounded(&bars[b ^ 1], (uint32_t)(((it + 1) >> 1) & 1));
            }
            return;
        }
        const BulkTile tl = bulk_tile(B, pt, k, lpre, lM, LW, t);
        const PrimeDev P = pick_prime(B, tl.tr);
        const typename A::Ctx L = A::ctx(P);
        uint64_t* __restrict__ d = dbuf[b];
        const double* __restrict__ tb = tbuf[b];
        const bool tab = TAB && tl.T != nullptr;
        const int esh = P.K - (k - lpre);
        const int S = P.S;
        const uint64_t smask = ((uint64_t)1 << S) - 1;
        const double* __restrict__ slo = reinterpret_cast<const double*>(INV ? P.slo_inv : P.slo_fwd);
        const double* __restrict__ shi = reinterpret_cast<const double*>(INV ? P.shi_inv : P.shi_fwd);
        auto twiddle = [&](typename A::T v, int m, int w) {
            if (tab) return A::twiddle(v, tb[(m << LW) + w], L);
            const uint64_t k1 = __brev((unsigned)m) >> (32 - LC);
            const uint64_t E = ((uint64_t)(tl.c0 + w) * k1) << esh;
            return A::twiddle(A::twiddle(v, __ldg(shi + (E >> S)), L), __ldg(slo + (E & smask)), L);
        };
        auto in = [&](int m, int w) -> typename A::T {
            const typename A::T v = A::ld(d[(m << LW) + w]);
            return INV ? twiddle(v, m, w) : v;
        };
        auto pre = [&](int m, int w) -> double { return tab ? tb[(m << LW) + w] : 0.0; };
        auto out = [&](int m, int w, typename A::T v, const double* tp) {
            if (!INV) v = (tp != nullptr && tab) ? A::twiddle(v, *tp, L) : twiddle(v, m, w);
            tl.base[((size_t)m << lM) + w] = A::st(v);
        };
        cols_fast_round<INV, LC, LW, RB, 0, A>(d, L, reinterpret_cast<const double*>(INV ? P.lvl_inv : P.lvl_fwd),
                                               in, out, pre);
        __syncthreads();  // buffer b is free again
        if (threadIdx.x < 32 && t + 2 * step < ntiles) {
            fence_async_smem();
            bulk_fetch<LC, LW>(bulk_tile(B, pt, k, lpre, lM, LW, t + 2 * step), lM, dbuf[b], tbuf[b], &bars[b]);
        }
    }
}

// The SplitSrc input written into `data` (for passes that read `data`).
__global__ void src_split_kernel(NttBatch B, int k)
{
    const size_t N = (size_t)1 << k;
    const size_t total = (size_t)B.count * N;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < total; g += (size_t)gridDim.x * blockDim.x) {
        const int tr = (int)(g >> k);
        const size_t j = g & (N - 1);
        const PrimeDev P = pick_prime(B, tr);
        const SrcRow r = src_row(B, tr);
        if (P.fp64) {
            B.data[(size_t)tr * B.stride + j] = dstore(dpiece56(src_piece56_raw(r.x, r.n, B.src.first + j), P.pd, P.pinv));
            continue;
        }
        const uint64_t v = src_piece_raw(B, r, j);
        B.data[(size_t)tr * B.stride + j] = P.lazy ? piece_to_strict(v, P.p) : v % P.p;
    }
}

static void materialize_src(const NttBatch& b, int k, cudaStream_t s)
{
    const size_t total = (size_t)b.count << k;
    ProfScope ps(KC_SPLIT, (4.0 + 8.0) * (double)total, s);
    src_split_kernel<<<grid_for(total, 256), 256, 0, s>>>(b, k);
    PIC_CHECK_LAUNCH();
    count_launch();
}

template <typename K>
static void set_smem(K kern, size_t smem)
{
    if (smem > 48 * 1024) PIC_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
}

// The fast kernels serve batches of lazy primes whose inner tables have order
// 2^13.  Passes run radix-8 rounds, or with rbits 4 radix-16 rounds for rows
// of 2^11 .. 2^13 points and columns of 2^8 .. 2^11 rows.
static bool fast_ok(const NttBatch& b, int k)
{
    const int rb = geom_of(b, k).rbits;
    if (!(PIC_NTT_FAST || b.prime[0].fp64) || (rb != 3 && rb != 4)) return false;
    for (int q = 0; q * b.per_prime < b.count; q++)
        if (!(b.prime[q].lazy || b.prime[q].fp64) || b.prime[q].fp64 != b.prime[0].fp64 || b.prime[q].IB != 13 ||
            b.prime[q].lvl_fwd == nullptr ||
            (q > 0 && (b.prime[q].slo_fwd == nullptr) != (b.prime[0].slo_fwd == nullptr)))
            return false;
    return true;
}

constexpr int fast_lrpc(int lr) { return lr < 11 ? 11 - lr : 0; }

template <bool INV, int LR, int RB, class A>
static void launch_rows_fast_t(const NttBatch& b, int k, cudaStream_t s)
{
    constexpr int LRPC = fast_lrpc(LR);
    using Sh = RowsFastShape<LR, LRPC, RB>;
    const size_t rows = (size_t)b.count << (k - LR);
    const size_t grid = (rows + ((size_t)1 << LRPC) - 1) >> LRPC;
    const size_t smem = sizeof(uint64_t) * Sh::TOT;
    set_smem(ntt_rows_fast_kernel<INV, LR, LRPC, RB, A>, smem);
    ntt_rows_fast_kernel<INV, LR, LRPC, RB, A><<<(unsigned)grid, Sh::NT, smem, s>>>(b, k);
}

template <bool INV, class A>
static bool launch_rows_fast(const NttBatch& b, int k, int lr, cudaStream_t s)
{
    if (!(lr == k || lr >= 11)) return false;
    if (geom_of(b, k).rbits == 4) {
        switch (lr) {
        case 11: launch_rows_fast_t<INV, 11, 4, A>(b, k, s); return true;
        case 12: launch_rows_fast_t<INV, 12, 4, A>(b, k, s); return true;
        case 13: launch_rows_fast_t<INV, 13, 4, A>(b, k, s); return true;
        default: break;  // shorter rows keep radix-8 rounds
        }
    }
    switch (lr) {
    case 1: launch_rows_fast_t<INV, 1, 3, A>(b, k, s); break;
    case 2: launch_rows_fast_t<INV, 2, 3, A>(b, k, s); break;
    case 3: launch_rows_fast_t<INV, 3, 3, A>(b, k, s); break;
    case 4: launch_rows_fast_t<INV, 4, 3, A>(b, k, s); break;
    case 5: launch_rows_fast_t<INV, 5, 3, A>(b, k, s); break;
    case 6: launch_rows_fast_t<INV, 6, 3, A>(b, k, s); break;
    case 7: launch_rows_fast_t<INV, 7, 3, A>(b, k, s); break;
    case 8: launch_rows_fast_t<INV, 8, 3, A>(b, k, s); break;
    case 9: launch_rows_fast_t<INV, 9, 3, A>(b, k, s); break;
    case 10: launch_rows_fast_t<INV, 10, 3, A>(b, k, s); break;
    case 11: launch_rows_fast_t<INV, 11, 3, A>(b, k, s); break;
    case 12: launch_rows_fast_t<INV, 12, 3, A>(b, k, s); break;
    case 13: launch_rows_fast_t<INV, 13, 3, A>(b, k, s); break;
    default: return false;
    }
    return true;
}

// Pass twiddle tables for root orders up to 2^kPassTableMaxBits (at most
// 6 x 16 x 2^24 bytes per order for the three product primes): built on the
// device on first use per (device, prime, direction, order, column height),
// kept for the process; never built while the stream is being captured (the
// pass then forms its twiddles from the two-level tables).  A table enters
// the cache only after its build kernel has finished (the building stream is
// synchronised), so a pass on any other stream that finds it in the cache
// reads a complete table.
constexpr int kPassTableMaxBits = 24;
static std::mutex g_pass_lock;
static std::map<std::tuple<int, uint64_t, int, int, int>, void*> g_pass_tables;

// FP64 column passes stream the per-point table only for blocks of at most
// 2^g_dbl_pass_bits points (tables that stay in L2); longer ones form each
// twiddle from the two-level tables (two products on the FP64 pipe, which
// has room), saving 16 bytes of DRAM traffic per point.
static int g_dbl_pass_bits = 20;
void ntt_set_dbl_pass_bits(int bits) { g_dbl_pass_bits = bits; }
int ntt_dbl_pass_bits() { return g_dbl_pass_bits; }

// Entries are Shoup pairs (16 bytes), or the twiddle w alone (8 bytes) for FP64 primes.
static const void* pass_table(const PrimeDev& P, bool inv, int lblock, int lc, cudaStream_t s)
{
    if (lblock > kPassTableMaxBits || (P.fp64 && lblock > g_dbl_pass_bits)) return nullptr;
    int dev = 0;
    PIC_CUDA(cudaGetDevice(&dev));
    const auto key = std::make_tuple(dev, P.p, inv ? 1 : 0, lblock, lc);
    std::lock_guard<std::mutex> g(g_pass_lock);
    auto it = g_pass_tables.find(key);
    if (it != g_pass_tables.end()) return it->second;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    PIC_CUDA(cudaStreamIsCapturing(s, &cs));
    if (cs != cudaStreamCaptureStatusNone) return nullptr;
    void* d = nullptr;
    if (raw_dev_alloc(&d, (P.fp64 ? sizeof(double) : sizeof(ulonglong2)) << lblock) != cudaSuccess)
        return nullptr;  // no room: the pass keeps the two-level tables
    const size_t n = (size_t)1 << lblock;
    pass_table_kernel<<<grid_for(n, 256), 256, 0, s>>>(d, P, inv ? 1 : 0, lblock, lc);
    PIC_CHECK_LAUNCH();
    count_launch();
    PIC_CUDA(cudaStreamSynchronize(s));  // complete before any other stream can find it
    g_pass_tables[key] = d;
    return d;
}

template <bool INV, int LC, int LW, int RB, class A>
static void launch_cols_fast_t(const NttBatch& b, int k, int lpre, size_t grid, cudaStream_t s)
{
    constexpr size_t smem = sizeof(uint64_t) << (LC + LW);
    PassTw pt{};
    bool all = true;
    for (int q = 0; q * b.per_prime < b.count; q++) {
        pt.t[q] = pass_table(b.prime[q], INV, k - lpre, LC, s);
        all = all && pt.t[q] != nullptr;
    }
    if (!all) pt = PassTw{};  // one form for every prime of the launch
    set_smem(ntt_cols_fast_kernel<INV, LC, LW, RB, A>, smem);
    ntt_cols_fast_kernel<INV, LC, LW, RB, A><<<(unsigned)grid, 256, smem, s>>>(b, k, lpre, pt);
}

template <bool INV, int LC, int RB, class A>
static bool launch_cols_fast_lc(const NttBatch& b, int k, int lpre, int lw, size_t grid, cudaStream_t s)
{
    switch (lw) {
    case 2: if constexpr (LC + 2 <= 13) { launch_cols_fast_t<INV, LC, 2, RB, A>(b, k, lpre, grid, s); return true; } break;
    case 3: if constexpr (LC + 3 <= 13) { launch_cols_fast_t<INV, LC, 3, RB, A>(b, k, lpre, grid, s); return true; } break;
    case 4: if constexpr (LC + 4 <= 13) { launch_cols_fast_t<INV, LC, 4, RB, A>(b, k, lpre, grid, s); return true; } break;
    case 5: if constexpr (LC + 5 <= 13) { launch_cols_fast_t<INV, LC, 5, RB, A>(b, k, lpre, grid, s); return true; } break;
    case 6: if constexpr (LC + 6 <= 13) { launch_cols_fast_t<INV, LC, 6, RB, A>(b, k, lpre, grid, s); return true; } break;
    default: break;
    }
    return false;
}

template <bool INV, class A>
static bool launch_cols_fast(const NttBatch& b, int k, int lpre, int lc, int lw, size_t grid, cudaStream_t s)
{
    if (geom_of(b, k).rbits == 4) {  // radix-16 rounds for the tall columns of long transforms
        switch (lc) {
        case 8: return launch_cols_fast_lc<INV, 8, 4, A>(b, k, lpre, lw, grid, s);
        case 9: return launch_cols_fast_lc<INV, 9, 4, A>(b, k, lpre, lw, grid, s);
        case 10: return launch_cols_fast_lc<INV, 10, 4, A>(b, k, lpre, lw, grid, s);
        case 11: return launch_cols_fast_lc<INV, 11, 4, A>(b, k, lpre, lw, grid, s);
        default: break;
        }
    }
    switch (lc) {
    case 1: return launch_cols_fast_lc<INV, 1, 3, A>(b, k, lpre, lw, grid, s);
    case 2: return launch_cols_fast_lc<INV, 2, 3, A>(b, k, lpre, lw, grid, s);
    case 3: return launch_cols_fast_lc<INV, 3, 3, A>(b, k, lpre, lw, grid, s);
    case 4: return launch_cols_fast_lc<INV, 4, 3, A>(b, k, lpre, lw, grid, s);
    case 5: return launch_cols_fast_lc<INV, 5, 3, A>(b, k, lpre, lw, grid, s);
    case 6: return launch_cols_fast_lc<INV, 6, 3, A>(b, k, lpre, lw, grid, s);
    case 7: return launch_cols_fast_lc<INV, 7, 3, A>(b, k, lpre, lw, grid, s);
    case 8: return launch_cols_fast_lc<INV, 8, 3, A>(b, k, lpre, lw, grid, s);
    case 9: return launch_cols_fast_lc<INV, 9, 3, A>(b, k, lpre, lw, grid, s);
    case 10: return launch_cols_fast_lc<INV, 10, 3, A>(b, k, lpre, lw, grid, s);
    case 11: return launch_cols_fast_lc<INV, 11, 3, A>(b, k, lpre, lw, grid, s);
    default: return false;
    }
}

// Column passes through the bulk-copy kernel (PIC_TUNE_COLS_BULK): FP64
// form, columns of 2^5 .. 2^9 rows, tiles 2^3 .. 2^6 columns wide, data
// 16-byte aligned with an even item stride.
// g_cols_bulk: 0 off, else log2 of the largest tile (points) the kernel
// takes; tiles are narrowed to it so that more CTAs share an SM.
static int g_cols_bulk = 0;
void ntt_set_cols_bulk(int bits) { g_cols_bulk = bits; }
int ntt_cols_bulk() { return g_cols_bulk; }

bool ntt_take_bulk_error()
{
    int e = 0, zero = 0;
    PIC_CUDA(cudaMemcpyFromSymbol(&e, g_ntt_bulk_error, sizeof e));
    if (e) PIC_CUDA(cudaMemcpyToSymbol(g_ntt_bulk_error, &zero, sizeof zero));
    return e != 0;
}

template <bool INV, int LC, int LW, int RB, bool TAB>
static bool launch_cols_bulk_tab(const NttBatch& b, int k, int lpre, const PassTw& pt, size_t ntiles, cudaStream_t s)
{
    auto kern = ntt_cols_bulk_kernel<INV, LC, LW, RB, TAB, ArithDbl>;
    constexpr size_t smem = BulkShape<LC, LW, TAB>::SMEM;
    set_smem(kern, smem);
    int per_sm = 0;
    PIC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, smem));
    if (per_sm < 1) return false;
    const size_t grid = std::min(ntiles, (size_t)ctx().num_sms * (size_t)per_sm);
    kern<<<(unsigned)grid, 256, smem, s>>>(b, k, lpre, pt, ntiles);
    return true;
}

template <bool INV, int LC, int LW, int RB>
static bool launch_cols_bulk_t(const NttBatch& b, int k, int lpre, size_t ntiles, cudaStream_t s)
{
    PassTw pt{};
    bool all = true;
    for (int q = 0; q * b.per_prime < b.count; q++) {
        pt.t[q] = pass_table(b.prime[q], INV, k - lpre, LC, s);
        all = all && pt.t[q] != nullptr;
    }
    if (!all) return launch_cols_bulk_tab<INV, LC, LW, RB, false>(b, k, lpre, PassTw{}, ntiles, s);
    return launch_cols_bulk_tab<INV, LC, LW, RB, true>(b, k, lpre, pt, ntiles, s);
}

template <bool INV, int LC, int RB>
static bool launch_cols_bulk_lc(const NttBatch& b, int k, int lpre, int lw, size_t ntiles, cudaStream_t s)
{
    switch (lw) {
    case 3: if constexpr (LC + 3 <= 12) return launch_cols_bulk_t<INV, LC, 3, RB>(b, k, lpre, ntiles, s); break;
    case 4: if constexpr (LC + 4 <= 12) return launch_cols_bulk_t<INV, LC, 4, RB>(b, k, lpre, ntiles, s); break;
    case 5: if constexpr (LC + 5 <= 12) return launch_cols_bulk_t<INV, LC, 5, RB>(b, k, lpre, ntiles, s); break;
    case 6: if constexpr (LC + 6 <= 12) return launch_cols_bulk_t<INV, LC, 6, RB>(b, k, lpre, ntiles, s); break;
    default: break;
    }
    return false;
}

template <bool INV>
static bool launch_cols_bulk(const NttBatch& b, int k, int lpre, int lc, int lw, size_t ntiles, cudaStream_t s)
{
    if (!g_cols_bulk || !b.prime[0].fp64 || b.src.words != nullptr || ((uintptr_t)b.data & 15) || (b.stride & 1))
        return false;
    if (lc + lw > g_cols_bulk) lw = g_cols_bulk - lc;
    if (lw < 3) return false;
    ntiles = (size_t)b.count << (k - lpre - lc - lw + lpre);  // tiles of the narrowed width
    if (geom_of(b, k).rbits == 4) {
        switch (lc) {
        case 8: return launch_cols_bulk_lc<INV, 8, 4>(b, k, lpre, lw, ntiles, s);
        case 9: return launch_cols_bulk_lc<INV, 9, 4>(b, k, lpre, lw, ntiles, s);
        default: break;
        }
    }
    switch (lc) {
    case 5: return launch_cols_bulk_lc<INV, 5, 3>(b, k, lpre, lw, ntiles, s);
    case 6: return launch_cols_bulk_lc<INV, 6, 3>(b, k, lpre, lw, ntiles, s);
    case 7: return launch_cols_bulk_lc<INV, 7, 3>(b, k, lpre, lw, ntiles, s);
    case 8: return launch_cols_bulk_lc<INV, 8, 3>(b, k, lpre, lw, ntiles, s);
    case 9: return launch_cols_bulk_lc<INV, 9, 3>(b, k, lpre, lw, ntiles, s);
    default: return false;
    }
}

template <bool INV>
static bool launch_rows_fast_any(const NttBatch& b, int k, int lr, cudaStream_t s)
{
    return b.prime[0].fp64 ? launch_rows_fast<INV, ArithDbl>(b, k, lr, s) : launch_rows_fast<INV, ArithInt>(b, k, lr, s);
}

template <bool INV>
static bool launch_cols_fast_any(const NttBatch& b, int k, int lpre, int lc, int lw, size_t grid, cudaStream_t s)
{
    return b.prime[0].fp64 ? launch_cols_fast<INV, ArithDbl>(b, k, lpre, lc, lw, grid, s)
                           : launch_cols_fast<INV, ArithInt>(b, k, lpre, lc, lw, grid, s);
}

static void launch_rows(bool inv, const NttBatch& b, int k, int lr, cudaStream_t s)
{
    if (fast_ok(b, k)) {
        ProfScope ps(KC_NTT_ROWS, 16.0 * (double)b.count * (double)((size_t)1 << k), s);
        if (inv ? launch_rows_fast_any<true>(b, k, lr, s) : launch_rows_fast_any<false>(b, k, lr, s)) {
            PIC_CHECK_LAUNCH();
            count_launch();
            return;
        }
    }
    PIC_REQUIRE(!b.prime[0].fp64, PIC_ERR_INVALID, "FP64 NTT row pass outside the fast kernels' shapes");
    if (!inv && b.src.words != nullptr) materialize_src(b, k, s);  // the general kernels read `data`
    int lrpc = 0;
    if (lr == k) {
        // several whole transforms per CTA when short, never straddling primes
        lrpc = 11 - lr;
        if (lrpc < 0) lrpc = 0;
        while (lrpc > 0 && (b.per_prime & ((1 << lrpc) - 1))) lrpc--;
    }
    const size_t rows = (size_t)b.count << (k - lr);
    const size_t grid = rows >> lrpc;
    ProfScope ps(KC_NTT_ROWS, 16.0 * (double)b.count * (double)((size_t)1 << k), s);
    const size_t smem = sizeof(uint64_t) << (lrpc + lr);
    const int rb = geom_of(b, k).rbits;
    int threads = 1 << (lrpc + lr - rb);
    if (threads < 32) threads = 32;
    if (threads > 512) threads = 512;
    const bool lazy = b.prime[0].lazy != 0;
#define PIC_ROWS(I, Z, R)                                                                        \
    do {                                                                                       \
        set_smem(ntt_rows_kernel<I, Z, R>, smem);                                              \
        ntt_rows_kernel<I, Z, R><<<(unsigned)grid, threads, smem, s>>>(b, k, lr, lrpc);        \
    } while (0)
    if (rb == 4) {
        if (inv) { if (lazy) PIC_ROWS(true, true, 4); else PIC_ROWS(true, false, 4); }
        else { if (lazy) PIC_ROWS(false, true, 4); else PIC_ROWS(false, false, 4); }
    } else if (rb == 2) {
        if (inv) { if (lazy) PIC_ROWS(true, true, 2); else PIC_ROWS(true, false, 2); }
        else { if (lazy) PIC_ROWS(false, true, 2); else PIC_ROWS(false, false, 2); }
    } else {
        if (inv) { if (lazy) PIC_ROWS(true, true, 3); else PIC_ROWS(true, false, 3); }
        else { if (lazy) PIC_ROWS(false, true, 3); else PIC_ROWS(false, false, 3); }
    }
#undef PIC_ROWS
    PIC_CHECK_LAUNCH();
    count_launch();
}

static void launch_cols(bool inv, const NttBatch& b, int k, int lpre, int lc, cudaStream_t s)
{
    const Geometry& gm = geom_of(b, k);
    int lw = gm.col_lw ? gm.col_lw : col_width_log2(lc);
    const int rb = gm.rbits;
    const int lM = k - lpre - lc;
    if (lc + lw > kInnerBits) lw = kInnerBits - lc;  // tile <= 2^13 points (64 KB)
    if (lw < 2) lw = 2;
    if (lw > lM) lw = lM;
    const size_t grid = (size_t)b.count << (lM - lw + lpre);
    const size_t smem = sizeof(uint64_t) << (lc + lw);
    ProfScope ps(KC_NTT_COLS, 16.0 * (double)b.count * (double)((size_t)1 << k), s);
    if (fast_ok(b, k) && b.prime[0].slo_fwd != nullptr &&
        (inv ? launch_cols_bulk<true>(b, k, lpre, lc, lw, grid, s) : launch_cols_bulk<false>(b, k, lpre, lc, lw, grid, s))) {
        PIC_CHECK_LAUNCH();
        count_launch();
        return;
    }
    if (fast_ok(b, k) && b.prime[0].slo_fwd != nullptr &&
        (inv ? launch_cols_fast_any<true>(b, k, lpre, lc, lw, grid, s)
             : launch_cols_fast_any<false>(b, k, lpre, lc, lw, grid, s))) {
        PIC_CHECK_LAUNCH();
        count_launch();
        return;
    }
    PIC_REQUIRE(!b.prime[0].fp64, PIC_ERR_INVALID, "FP64 NTT column pass outside the fast kernels' shapes");
    if (!inv && b.src.words != nullptr) materialize_src(b, k, s);  // the general kernels read `data`
    const bool lazy = b.prime[0].lazy != 0;
#define PIC_COLS(I, Z, R)                                                                          \
    do {                                                                                         \
        set_smem(ntt_cols_kernel<I, Z, R>, smem);                                                \
        ntt_cols_kernel<I, Z, R><<<(unsigned)grid, 256, smem, s>>>(b, k, lpre, lc, lw);          \
    } while (0)
    if (rb == 4) {
        if (inv) { if (lazy) PIC_COLS(true, true, 4); else PIC_COLS(true, false, 4); }
        else { if (lazy) PIC_COLS(false, true, 4); else PIC_COLS(false, false, 4); }
    } else if (rb == 2) {
        if (inv) { if (lazy) PIC_COLS(true, true, 2); else PIC_COLS(true, false, 2); }
        else { if (lazy) PIC_COLS(false, true, 2); else PIC_COLS(false, false, 2); }
    } else {
        if (inv) { if (lazy) PIC_COLS(true, true, 3); else PIC_COLS(true, false, 3); }
        else { if (lazy) PIC_COLS(false, true, 3); else PIC_COLS(false, false, 3); }
    }
#undef PIC_COLS
    PIC_CHECK_LAUNCH();
    count_launch();
}

static void check_batch(const NttBatch& b, int k)
{
    PIC_REQUIRE(k >= 1 && k <= 32, PIC_ERR_INVALID, "NTT length out of range");
    PIC_REQUIRE(b.count > 0 && b.per_prime > 0 && b.count <= b.per_prime * kMaxPrimesPerBatch,
                PIC_ERR_INVALID, "bad NTT batch");
    PIC_REQUIRE(b.stride >= ((size_t)1 << k), PIC_ERR_INVALID, "NTT batch stride too small");
    for (int q = 0; q * b.per_prime < b.count; q++) {
        PIC_REQUIRE(b.prime[q].K >= k, PIC_ERR_INVALID, "prime has no root of unity of this order");
        PIC_REQUIRE(b.prime[q].lazy == b.prime[0].lazy && b.prime[q].fp64 == b.prime[0].fp64, PIC_ERR_INVALID,
                    "mixed prime kinds in one batch");
    }
}

void ntt_forward_dif(const NttBatch& b, int k, cudaStream_t s)
{
    check_batch(b, k);
    std::vector<int> bits = ntt_pass_bits(k, b.prime[0].fp64 ? kFormDbl : kFormInt);
    NttBatch rest = b;
    rest.src = SplitSrc{};  // only the first pass reads the child slots
    int lpre = 0;
    for (size_t i = 0; i + 1 < bits.size(); i++) {
        launch_cols(false, i == 0 ? b : rest, k, lpre, bits[i], s);
        lpre += bits[i];
    }
    launch_rows(false, bits.size() == 1 ? b : rest, k, bits.back(), s);
}

void ntt_inverse_dit(const NttBatch& b_in, int k, cudaStream_t s)
{
    NttBatch b = b_in;
    b.src = SplitSrc{};
    check_batch(b, k);
    std::vector<int> bits = ntt_pass_bits(k, b.prime[0].fp64 ? kFormDbl : kFormInt);
    launch_rows(true, b, k, bits.back(), s);
    int lpre = k - bits.back();
    for (int i = (int)bits.size() - 2; i >= 0; i--) {
        lpre -= bits[i];
        launch_cols(true, b, k, lpre, bits[i], s);
    }
}

__global__ void bitreverse_kernel(NttBatch B, int k)
{
    const size_t n = (size_t)1 << k;
    const size_t total = (size_t)B.count * n;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < total;
         g += (size_t)gridDim.x * blockDim.x) {
        const size_t tr = g >> k, i = g & (n - 1);
        const size_t j = __brevll(i) >> (64 - k);
        if (i < j) {
            uint64_t* d = B.data + tr * B.stride;
            uint64_t t = d[i];
            d[i] = d[j];
            d[j] = t;
        }
    }
}

void ntt_bitreverse(const NttBatch& b, int k, cudaStream_t s)
{
    const size_t total = (size_t)b.count << k;
    bitreverse_kernel<<<grid_for(total, 256), 256, 0, s>>>(b, k);
    PIC_CHECK_LAUNCH();
    count_launch();
}

__global__ void pointwise_mont_kernel(NttBatch B, const uint64_t* __restrict__ other, size_t ostride, int k)
{
    const size_t n = (size_t)1 << k;
    const size_t total = (size_t)B.count * n;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < total;
         g += (size_t)gridDim.x * blockDim.x) {
        const size_t tr = g >> k, i = g & (n - 1);
        const PrimeDev P = pick_prime(B, (int)tr);
        uint64_t* d = B.data + tr * B.stride + i;
        if (P.fp64) {  // forward outputs |x| <= p: the product is below p^2
            *d = dstore(dmul_mod(dbits(*d), dbits(other[tr * ostride + i]), P.pd, P.pinv));
            continue;
        }
        *d = P.lazy ? mont_mul_c(*d, other[tr * ostride + i], P.p, (uint32_t)(P.p >> 32))
                    : mont_mul(*d, other[tr * ostride + i], P.p, P.pinv_neg);
    }
}

void ntt_pointwise_mont(const NttBatch& a, const uint64_t* b, int k, cudaStream_t s, size_t b_stride)
{
    const size_t total = (size_t)a.count << k;
    ProfScope ps(KC_NTT_POINTWISE, 24.0 * (double)total, s);
    pointwise_mont_kernel<<<grid_for(total, 256), 256, 0, s>>>(a, b, b_stride ? b_stride : a.stride, k);
    PIC_CHECK_LAUNCH();
    count_launch();
}

__global__ void pointwise_plain_kernel(uint64_t* T, const uint64_t* A, size_t n, uint64_t p,
                                       uint64_t pinv_neg, uint64_t r2)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        T[i] = mont_mul(mont_mul(T[i], A[i], p, pinv_neg), r2, p, pinv_neg);
}

void ntt_pointwise_plain(uint64_t* T, const uint64_t* A, int k, const PrimeDev& P, cudaStream_t s)
{
    const size_t n = (size_t)1 << k;
    pointwise_plain_kernel<<<grid_for(n, 256), 256, 0, s>>>(T, A, n, P.p, P.pinv_neg, P.r2);
    PIC_CHECK_LAUNCH();
    count_launch();
}

__global__ void scale_kernel(uint64_t* T, size_t n, uint64_t c_mont, uint64_t p, uint64_t pinv_neg)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        T[i] = mont_mul(T[i], c_mont, p, pinv_neg);
}

void ntt_scale_ninv(uint64_t* T, int k, const PrimeDev& P, cudaStream_t s)
{
    const size_t n = (size_t)1 << k;
    const uint64_t ninv = host_powmod(n % P.p, P.p - 2, P.p);
    scale_kernel<<<grid_for(n, 256), 256, 0, s>>>(T, n, to_mont(ninv, P.p), P.p, P.pinv_neg);
    PIC_CHECK_LAUNCH();
    count_launch();
}

}  // namespace pic
