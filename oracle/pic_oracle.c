/* pic_oracle.c -- plain-C restatement of Piculator's multiply path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the thing measured or shipped).
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * the library built from this file.
 *
 * Each function names the reference lines it restates.  The reference is
 * MSVC C++ (BigFloat.cpp, NTT.cpp, FFT.cpp, PI.h); the semantics below --
 * truncation windows, carry rules, seeds, sizes -- are reproduced exactly,
 * while the arithmetic inside a product is free to differ because every
 * product is exact (BigFloat.cpp:413-487 forms the full product of the
 * truncated operands).
 */
#define _GNU_SOURCE
#include "pic_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

/* ------------------------------------------------------------------------ */
/* BigFloat value (BigFloat.h:32-36).  T is malloc-owned.                    */

typedef struct {
    int sign;       /* 1 = positive or zero */
    int64_t exp;
    size_t L;
    uint32_t* T;
} bf;

static bf bf_zero(void)
{
    bf z = {1, 0, 0, NULL};
    return z;
}

static void bf_free(bf* x)
{
    free(x->T);
    x->T = NULL;
    x->L = 0;
}

static void* xmalloc(size_t n)
{
    void* p = malloc(n ? n : 1);
    if (!p) {
        fprintf(stderr, "pic_oracle: out of memory (%zu bytes)\n", n);
        abort();
    }
    return p;
}

/* BigFloat(uint32_t x, bool sign) -- BigFloat.cpp:64-79 */
static bf bf_from_u32(uint32_t x, int sign)
{
    bf z = bf_zero();
    if (x == 0) return z;
    z.sign = sign;
    z.L = 1;
    z.T = (uint32_t*)xmalloc(sizeof(uint32_t));
    z.T[0] = x;
    return z;
}

/* negate -- BigFloat.cpp:150-155 */
static void bf_negate(bf* x)
{
    if (x->L == 0) return;
    x->sign = !x->sign;
}

/* word_at -- BigFloat.cpp:109-122 */
static uint32_t bf_word_at(const bf* x, int64_t mag)
{
    if (mag < x->exp) return 0;
    if (mag >= x->exp + (int64_t)x->L) return 0;
    return x->T[(size_t)(mag - x->exp)];
}

/* ucmp -- BigFloat.cpp:123-147 */
static int bf_ucmp(const bf* a, const bf* x)
{
    int64_t magA = a->exp + (int64_t)a->L;
    int64_t magB = x->exp + (int64_t)x->L;
    if (magA > magB) return 1;
    if (magA < magB) return -1;
    int64_t mag = magA;
    while (mag >= a->exp || mag >= x->exp) {
        uint32_t wa = bf_word_at(a, mag), wb = bf_word_at(x, mag);
        if (wa < wb) return -1;
        if (wa > wb) return 1;
        mag--;
    }
    return 0;
}

/* mul(uint32_t) -- BigFloat.cpp:156-183 */
static bf bf_mul_u32(const bf* a, uint32_t x)
{
    if (a->L == 0 || x == 0) return bf_zero();
    bf z;
    z.sign = a->sign;
    z.exp = a->exp;
    z.L = a->L;
    z.T = (uint32_t*)xmalloc(sizeof(uint32_t) * (z.L + 1));
    uint64_t carry = 0;
    for (size_t c = 0; c < a->L; c++) {
        carry += (uint64_t)a->T[c] * x;
        z.T[c] = (uint32_t)carry;
        carry >>= 32;
    }
    if (carry != 0) z.T[z.L++] = (uint32_t)carry;
    return z;
}

#define EXTRA_PRECISION 2 /* YCL_BIGFLOAT_EXTRA_PRECISION, BigFloat.h:6 */

/* uadd -- BigFloat.cpp:184-232.  Each addend is read only inside the window
 * [bot, top); words below it are dropped before adding (their carry is lost). */
static bf bf_uadd(const bf* a, const bf* x, size_t p)
{
    int64_t magA = a->exp + (int64_t)a->L;
    int64_t magB = x->exp + (int64_t)x->L;
    int64_t top = magA > magB ? magA : magB;
    int64_t bot = a->exp < x->exp ? a->exp : x->exp;
    int64_t TL = top - bot;
    if (p == 0) p = (size_t)TL;
    else p += EXTRA_PRECISION;
    if (TL > (int64_t)p) {
        bot = top - (int64_t)p;
        TL = (int64_t)p;
    }
    bf z;
    z.sign = a->sign;
    z.exp = bot;
    z.L = (uint32_t)TL;
    z.T = (uint32_t*)xmalloc(sizeof(uint32_t) * (z.L + 1));
    uint32_t carry = 0;
    for (size_t c = 0; bot < top; bot++, c++) {
        uint64_t s = (uint64_t)bf_word_at(a, bot) + bf_word_at(x, bot) + carry;
        z.T[c] = (uint32_t)s;
        carry = (uint32_t)(s >> 32);
    }
    if (carry != 0) z.T[z.L++] = 1;
    return z;
}

/* usub -- BigFloat.cpp:233-287 (requires |a| >= |x|) */
static bf bf_usub(const bf* a, const bf* x, size_t p)
{
    int64_t magA = a->exp + (int64_t)a->L;
    int64_t magB = x->exp + (int64_t)x->L;
    int64_t top = magA > magB ? magA : magB;
    int64_t bot = a->exp < x->exp ? a->exp : x->exp;
    int64_t TL = top - bot;
    if (p == 0) p = (size_t)TL;
    else p += EXTRA_PRECISION;
    if (TL > (int64_t)p) {
        bot = top - (int64_t)p;
        TL = (int64_t)p;
    }
    bf z;
    z.sign = a->sign;
    z.exp = bot;
    z.L = (uint32_t)TL;
    z.T = (uint32_t*)xmalloc(sizeof(uint32_t) * (z.L ? z.L : 1));
    uint32_t borrow = 0;
    for (size_t c = 0; bot < top; bot++, c++) {
        uint64_t d = (uint64_t)bf_word_at(a, bot) - bf_word_at(x, bot) - borrow;
        z.T[c] = (uint32_t)d;
        borrow = (uint32_t)(d >> 63);
    }
    while (z.L > 0 && z.T[z.L - 1] == 0) z.L--;
    if (z.L == 0) {
        z.exp = 0;
        z.sign = 1;
        free(z.T);
        z.T = NULL;
    }
    return z;
}

/* add -- BigFloat.cpp:288-305 */
static bf bf_add(const bf* a, const bf* x, size_t p)
{
    if (a->sign == x->sign) return bf_uadd(a, x, p);
    if (bf_ucmp(a, x) > 0) return bf_usub(a, x, p);
    return bf_usub(x, a, p);
}

/* sub -- BigFloat.cpp:306-325 */
static bf bf_sub(const bf* a, const bf* x, size_t p)
{
    if (a->sign != x->sign) return bf_uadd(a, x, p);
    if (bf_ucmp(a, x) > 0) return bf_usub(a, x, p);
    bf z = bf_usub(x, a, p);
    bf_negate(&z);
    return z;
}

/* ------------------------------------------------------------------------ */
/* Modular arithmetic and the reference's prime table (NTT.cpp:85-158).      */

static uint64_t mulmod(uint64_t a, uint64_t b, uint64_t p)
{
    return (uint64_t)(((u128)a * b) % p);
}

static uint64_t powmod(uint64_t a, uint64_t e, uint64_t p)
{
    uint64_t r = 1;
    a %= p;
    while (e) {
        if (e & 1) r = mulmod(r, a, p);
        a = mulmod(a, a, p);
        e >>= 1;
    }
    return r;
}

/* primes map -- NTT.cpp:125-158 (same table: the transform length selects the
 * prime, so a drop-in must use identical values). */
static const uint64_t k_primes[43] = {
    [11] = 9223372036854675457ull, [12] = 9223372036854497281ull,
    [13] = 9223372036854497281ull, [14] = 9223372036854497281ull,
    [15] = 9223372036853661697ull, [16] = 9223372036853661697ull,
    [17] = 9223372036844421121ull, [18] = 9223372036836950017ull,
    [19] = 9223372036836950017ull, [20] = 9223372036836950017ull,
    [21] = 9223372036752015361ull, [22] = 9223372036737335297ull,
    [23] = 9223372036737335297ull, [24] = 9223372036737335297ull,
    [25] = 9223372036083023873ull, [26] = 9223372035915251713ull,
    [27] = 9223372035915251713ull, [28] = 9223372034170421249ull,
    [29] = 9223372034170421249ull, [30] = 9223372006790004737ull,
    [31] = 9223372006790004737ull, [32] = 9223372006790004737ull,
    [33] = 9223371564408373249ull, [34] = 9223371280940531713ull,
    [35] = 9223371280940531713ull, [36] = 9223371280940531713ull,
    [37] = 9223369837831520257ull, [38] = 9223369837831520257ull,
    [39] = 9223369837831520257ull, [40] = 9223369837831520257ull,
    [41] = 9223369837831520257ull, [42] = 9223341250529198081ull,
};

uint64_t oracle_prime(int k)
{
    if (k < 11) k = 11;
    if (k > 42) return 0;
    return k_primes[k];
}

/* generator -- NTT.cpp:104-123: smallest g >= 2 whose order is p-1, found
 * by trial-division factoring of p-1. */
uint64_t oracle_generator(uint64_t p)
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
        int ok = 1;
        for (int i = 0; i < nf && ok; ++i) ok &= powmod(g, phi / fact[i], p) != 1;
        if (ok) return g;
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* NTT (NNT::init NTT.cpp:169-188, NTT_fast :191-223, iNTT :80-84).          */
/* Natural-order DFT X_j = sum x_i w^(ij) mod p with w = g^((p-1)/n).        */
/* Iterative radix-2 with Montgomery multiplication; same transform, no      */
/* reorder passes.                                                          */

typedef struct {
    uint64_t p, pinv_neg, r2; /* -p^-1 mod 2^64, 2^128 mod p */
} mont_t;

static mont_t mont_make(uint64_t p)
{
    mont_t m;
    m.p = p;
    uint64_t inv = p; /* Newton iteration for p^-1 mod 2^64 */
    for (int i = 0; i < 6; i++) inv *= 2 - p * inv;
    m.pinv_neg = (uint64_t)0 - inv;
    u128 r = ((u128)1 << 64) % p;
    m.r2 = (uint64_t)((r * r) % p);
    return m;
}

static inline uint64_t mont_mul(const mont_t* m, uint64_t a, uint64_t b)
{
    u128 t = (u128)a * b;
    uint64_t q = (uint64_t)t * m->pinv_neg;
    u128 u = t + (u128)q * m->p; /* a, b < p < 2^63: no overflow */
    uint64_t r = (uint64_t)(u >> 64);
    return r >= m->p ? r - m->p : r;
}

static inline uint64_t mont_in(const mont_t* m, uint64_t a) { return mont_mul(m, a, m->r2); }
static inline uint64_t mont_out(const mont_t* m, uint64_t a) { return mont_mul(m, a, 1); }

static void ntt_core(uint64_t* a, size_t n, uint64_t w, uint64_t p)
{
    mont_t m = mont_make(p);
    /* bit-reversal permutation */
    for (size_t i = 1, j = 0; i < n; i++) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            uint64_t t = a[i];
            a[i] = a[j];
            a[j] = t;
        }
    }
    for (size_t i = 0; i < n; i++) a[i] = mont_in(&m, a[i]);
    uint64_t* tw = (uint64_t*)xmalloc(sizeof(uint64_t) * (n / 2 + 1));
    for (size_t len = 2; len <= n; len <<= 1) {
        uint64_t wl = mont_in(&m, powmod(w, n / len, p));
        size_t half = len / 2;
        tw[0] = mont_in(&m, 1);
        for (size_t j = 1; j < half; j++) tw[j] = mont_mul(&m, tw[j - 1], wl);
        for (size_t i = 0; i < n; i += len)
            for (size_t j = 0; j < half; j++) {
                uint64_t u = a[i + j];
                uint64_t v = mont_mul(&m, a[i + j + half], tw[j]);
                uint64_t s = u + v;
                a[i + j] = s >= p ? s - p : s;
                a[i + j + half] = u >= v ? u - v : u + p - v;
            }
    }
    free(tw);
    for (size_t i = 0; i < n; i++) a[i] = mont_out(&m, a[i]);
}

int oracle_ntt(int k, int inverse, uint64_t* data, uint64_t* p_out, uint64_t* g_out,
               uint64_t* w_out)
{
    if (k < 1 || k > 42) return -1;
    uint64_t p = oracle_prime(k);
    uint64_t g = oracle_generator(p);
    uint64_t n = (uint64_t)1 << k;
    uint64_t L = (p - 1) / n;
    uint64_t w = powmod(g, L, p);              /* W  = r^L       NTT.cpp:183 */
    uint64_t iw = powmod(g, p - 1 - L, p);     /* iW = r^(p-1-L) NTT.cpp:184 */
    ntt_core(data, (size_t)n, inverse ? iw : w, p);
    if (inverse) {
        uint64_t rn = powmod(n % p, p - 2, p); /* rN = n^(p-2)   NTT.cpp:185 */
        for (uint64_t i = 0; i < n; i++) data[i] = mulmod(data[i], rn, p);
    }
    if (p_out) *p_out = p;
    if (g_out) *g_out = g;
    if (w_out) *w_out = inverse ? iw : w;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* FFT (FFT.cpp:31-463): forward DIF with exp(+i 2 pi c / 2^s) twiddles,     */
/* natural in / bit-reversed out; inverse DIT with the conjugate twiddles,  */
/* bit-reversed in / natural out, unscaled.                                 */

static void fft_twiddles(double* tw, size_t n)
{
    /* tw[2c], tw[2c+1] = cos, sin(2 pi c / n), c < n/2 -- the table of
     * fft_ensure_table, FFT.cpp:45-56 */
    double omega = 2 * 3.14159265358979323846 / (double)n; /* M_PI, FFT.cpp:21 */
    for (size_t c = 0; c < n / 2; c++) {
        tw[2 * c] = cos(omega * (double)c);
        tw[2 * c + 1] = sin(omega * (double)c);
    }
}

static void fft_dif_forward(double* a, size_t n, const double* tw)
{
    for (size_t len = n; len >= 2; len >>= 1) {
        size_t half = len / 2, stride = n / len;
        for (size_t i = 0; i < n; i += len)
            for (size_t j = 0; j < half; j++) {
                double* x = a + 2 * (i + j);
                double* y = a + 2 * (i + j + half);
                double wr = tw[2 * j * stride], wi = tw[2 * j * stride + 1];
                double ar = x[0] + y[0], ai = x[1] + y[1];
                double dr = x[0] - y[0], di = x[1] - y[1];
                x[0] = ar;
                x[1] = ai;
                y[0] = dr * wr - di * wi;
                y[1] = dr * wi + di * wr;
            }
    }
}

static void fft_dit_inverse(double* a, size_t n, const double* tw)
{
    for (size_t len = 2; len <= n; len <<= 1) {
        size_t half = len / 2, stride = n / len;
        for (size_t i = 0; i < n; i += len)
            for (size_t j = 0; j < half; j++) {
                double* x = a + 2 * (i + j);
                double* y = a + 2 * (i + j + half);
                double wr = tw[2 * j * stride], wi = -tw[2 * j * stride + 1];
                double br = y[0] * wr - y[1] * wi, bi = y[0] * wi + y[1] * wr;
                double xr = x[0], xi = x[1];
                x[0] = xr + br;
                x[1] = xi + bi;
                y[0] = xr - br;
                y[1] = xi - bi;
            }
    }
}

int oracle_fft(int k, int op, double* data)
{
    if (k < 1 || k > 30) return -1;
    size_t n = (size_t)1 << k;
    double* tw = (double*)xmalloc(sizeof(double) * n);
    fft_twiddles(tw, n);
    if (op == 0) fft_dif_forward(data, n, tw);
    else fft_dit_inverse(data, n, tw);
    free(tw);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Exact product engines.                                                   */

static int g_mode = ORACLE_MODE_AUTO;
static double g_fft_last_err = 0.0;
static uint64_t g_fft_recomputes = 0;

void oracle_set_mode(int mode) { g_mode = mode; }
int oracle_get_mode(void) { return g_mode; }
double oracle_fft_last_max_err(void) { return g_fft_last_err; }
uint64_t oracle_fft_recomputes(void) { return g_fft_recomputes; }

static void mul_school(const uint32_t* a, size_t na, const uint32_t* b, size_t nb, uint32_t* z)
{
    memset(z, 0, sizeof(uint32_t) * (na + nb));
    for (size_t i = 0; i < na; i++) {
        uint64_t carry = 0, ai = a[i];
        for (size_t j = 0; j < nb; j++) {
            carry += ai * b[j] + z[i + j];
            z[i + j] = (uint32_t)carry;
            carry >>= 32;
        }
        z[i + nb] = (uint32_t)carry;
    }
}

/* int_to_ntt (NTT.cpp:330-341) + forward/pointwise/inverse (NTT.cpp:306-328)
 * + ntt_to_int (NTT.cpp:343-369): 16-bit points, length 2^k >= 4 (na+nb)
 * (BigFloat.cpp:380-385), the reference's prime for k. */
static void mul_ntt(const uint32_t* a, size_t na, const uint32_t* b, size_t nb, uint32_t* z)
{
    size_t zl = na + nb;
    int k = 0;
    size_t n = 1;
    while (n < 4 * zl) {
        n <<= 1;
        k++;
    }
    if (k < 11) {
        k = 11;
        n = (size_t)1 << 11;
    }
    uint64_t* ta = (uint64_t*)calloc(n, sizeof(uint64_t));
    uint64_t* tb = (uint64_t*)calloc(n, sizeof(uint64_t));
    if (!ta || !tb) abort();
    for (size_t i = 0; i < na; i++) {
        ta[2 * i] = a[i] & 0xffff;
        ta[2 * i + 1] = a[i] >> 16;
    }
    for (size_t i = 0; i < nb; i++) {
        tb[2 * i] = b[i] & 0xffff;
        tb[2 * i + 1] = b[i] >> 16;
    }
    uint64_t p;
    oracle_ntt(k, 0, ta, &p, NULL, NULL);
    oracle_ntt(k, 0, tb, NULL, NULL, NULL);
    for (size_t i = 0; i < n; i++) ta[i] = mulmod(ta[i], tb[i], p);
    oracle_ntt(k, 1, ta, NULL, NULL, NULL);
    uint64_t carry = 0;
    for (size_t c = 0; c < zl; c++) {
        uint32_t word;
        carry += ta[2 * c];
        word = (uint32_t)(carry & 0xffff);
        carry >>= 16;
        carry += ta[2 * c + 1];
        word |= (uint32_t)(carry & 0xffff) << 16;
        carry >>= 16;
        z[c] = word;
    }
    free(ta);
    free(tb);
}

/* int_to_fft (FFT.cpp:485-519) + forward/pointwise/inverse + fft_to_int
 * (FFT.cpp:520-571): four 8-bit real points per word, length 2^k >= 4 (na+nb),
 * round half up after scaling by 2^-k.  Returns the max rounding distance. */
static double mul_fft(const uint32_t* a, size_t na, const uint32_t* b, size_t nb, uint32_t* z)
{
    size_t zl = na + nb;
    size_t n = 1;
    while (n < 4 * zl) n <<= 1;
    double* ta = (double*)calloc(2 * n, sizeof(double));
    double* tb = (double*)calloc(2 * n, sizeof(double));
    double* tw = (double*)xmalloc(sizeof(double) * n);
    if (!ta || !tb) abort();
    for (size_t i = 0; i < na; i++)
        for (int q = 0; q < 4; q++) ta[2 * (4 * i + q)] = (double)((a[i] >> (8 * q)) & 0xff);
    for (size_t i = 0; i < nb; i++)
        for (int q = 0; q < 4; q++) tb[2 * (4 * i + q)] = (double)((b[i] >> (8 * q)) & 0xff);
    fft_twiddles(tw, n);
    fft_dif_forward(ta, n, tw);
    fft_dif_forward(tb, n, tw);
    for (size_t i = 0; i < n; i++) { /* fft_pointwise, FFT.cpp:464-484 */
        double ar = ta[2 * i], ai = ta[2 * i + 1], br = tb[2 * i], bi = tb[2 * i + 1];
        ta[2 * i] = ar * br - ai * bi;
        ta[2 * i + 1] = ar * bi + ai * br;
    }
    fft_dit_inverse(ta, n, tw);
    double scale = 1.0 / (double)n, maxerr = 0.0;
    uint64_t carry = 0;
    for (size_t c = 0; c < zl; c++) {
        uint32_t word = 0;
        for (int q = 0; q < 4; q++) {
            double f = ta[2 * (4 * c + q)] * scale;
            double r = floor(f + 0.5);
            double e = fabs(f - r);
            if (e > maxerr) maxerr = e;
            carry += (uint64_t)(f + 0.5);
            word |= (uint32_t)(carry & 0xff) << (8 * q);
            carry >>= 8;
        }
        z[c] = word;
    }
    free(ta);
    free(tb);
    free(tw);
    return maxerr;
}

void oracle_mul_words(const uint32_t* a, size_t na, const uint32_t* b, size_t nb, uint32_t* z)
{
    size_t zl = na + nb;
    int mode = g_mode;
    if (mode == ORACLE_MODE_AUTO) {
        size_t mn = na < nb ? na : nb;
        if (mn <= 40 || (double)na * (double)nb <= 4096.0) mode = ORACLE_MODE_SCHOOL;
        else {
            size_t n = 1;
            int k = 0;
            while (n < 4 * zl) {
                n <<= 1;
                k++;
            }
            mode = k < 27 ? ORACLE_MODE_FFT : ORACLE_MODE_NTT; /* BigFloat.cpp:386 */
        }
    }
    if (mode == ORACLE_MODE_SCHOOL) {
        mul_school(a, na, b, nb, z);
    } else if (mode == ORACLE_MODE_FFT) {
        double e = mul_fft(a, na, b, nb, z);
        g_fft_last_err = e;
        if (e > 0.25) { /* rounding too close to call: recompute exactly */
            g_fft_recomputes++;
            mul_ntt(a, na, b, nb, z);
        }
    } else {
        mul_ntt(a, na, b, nb, z);
    }
}

/* mul(const BigFloat&, p) -- BigFloat.cpp:326-444 */
static bf bf_mul(const bf* a, const bf* x, size_t p)
{
    if (a->L == 0 || x->L == 0) return bf_zero();
    if (p == 0) p = a->L + x->L;
    else p += EXTRA_PRECISION;
    int64_t Aexp = a->exp, Bexp = x->exp;
    size_t AL = a->L, BL = x->L;
    const uint32_t* AT = a->T;
    const uint32_t* BT = x->T;
    if (AL > p) {
        size_t chop = AL - p;
        AL = p;
        Aexp += (int64_t)chop;
        AT += chop;
    }
    if (BL > p) {
        size_t chop = BL - p;
        BL = p;
        Bexp += (int64_t)chop;
        BT += chop;
    }
    bf z;
    z.sign = a->sign == x->sign;
    z.exp = Aexp + Bexp;
    z.L = AL + BL;
    z.T = (uint32_t*)xmalloc(sizeof(uint32_t) * z.L);
    oracle_mul_words(AT, AL, BT, BL, z.T);
    if (z.T[z.L - 1] == 0) z.L--; /* BigFloat.cpp:411-412, :436-437 */
    return z;
}

/* rcp -- BigFloat.cpp:445-511 */
static int bf_rcp(const bf* a, size_t p, bf* out)
{
    if (a->L == 0) return -2; /* throw "Divide by Zero" */
    if (p == 0) {
        int64_t Aexp = a->exp;
        size_t AL = a->L;
        const uint32_t* AT = a->T;
        if (AL > 3) {
            size_t chop = AL - 3;
            AL = 3;
            Aexp += (int64_t)chop;
            AT += chop;
        }
        double val = (double)AT[0];
        if (AL >= 2) val += (double)AT[1] * 4294967296.;
        if (AL >= 3) val += (double)AT[2] * 4294967296. * 4294967296.;
        val = 1. / val;
        Aexp = -Aexp;
        while (val < 4294967296.) {
            val *= 4294967296.;
            Aexp--;
        }
        uint64_t v = (uint64_t)val;
        bf o;
        o.sign = a->sign;
        o.T = (uint32_t*)xmalloc(2 * sizeof(uint32_t));
        o.T[0] = (uint32_t)v;
        o.T[1] = (uint32_t)(v >> 32);
        o.L = 2;
        o.exp = Aexp;
        *out = o;
        return 0;
    }
    size_t s = p / 2 + 1;
    if (p == 1) s = 0;
    if (p == 2) s = 1;
    bf T;
    int rc = bf_rcp(a, s, &T);
    if (rc) return rc;
    /* r1 = r0 - (r0 * x - 1) * r0 -- BigFloat.cpp:510 */
    bf one = bf_from_u32(1, 1);
    bf t1 = bf_mul(a, &T, p);
    bf t2 = bf_sub(&t1, &one, p);
    bf t3 = bf_mul(&t2, &T, p);
    *out = bf_sub(&T, &t3, p);
    bf_free(&one);
    bf_free(&t1);
    bf_free(&t2);
    bf_free(&t3);
    bf_free(&T);
    return 0;
}

/* invsqrt -- BigFloat.cpp:516-568 */
static int bf_invsqrt(uint32_t x, size_t p, bf* out)
{
    if (x == 0) return -2;
    if (p == 0) {
        double val = 1. / sqrt((double)x);
        int64_t e = 0;
        while (val < 4294967296.) {
            val *= 4294967296.;
            e--;
        }
        uint64_t v = (uint64_t)val;
        bf o;
        o.sign = 1;
        o.T = (uint32_t*)xmalloc(2 * sizeof(uint32_t));
        o.T[0] = (uint32_t)v;
        o.T[1] = (uint32_t)(v >> 32);
        o.L = 2;
        o.exp = e;
        *out = o;
        return 0;
    }
    size_t s = p / 2 + 1;
    if (p == 1) s = 0;
    if (p == 2) s = 1;
    bf T;
    int rc = bf_invsqrt(x, s, &T);
    if (rc) return rc;
    bf xb = bf_from_u32(x, 1), one = bf_from_u32(1, 1);
    bf t1 = bf_mul(&T, &T, p);        /* r0^2 */
    bf t2 = bf_mul(&t1, &xb, 0);      /* r0^2 * x, full BigFloat mul with p = 0 */
    bf t3 = bf_sub(&t2, &one, p);     /* r0^2 * x - 1 */
    bf t4 = bf_mul_u32(&t3, 2147483648u);
    t4.exp--;                         /* (r0^2 * x - 1) / 2 */
    bf t5 = bf_mul(&t4, &T, p);
    *out = bf_sub(&T, &t5, p);
    bf_free(&xb);
    bf_free(&one);
    bf_free(&t1);
    bf_free(&t2);
    bf_free(&t3);
    bf_free(&t4);
    bf_free(&t5);
    bf_free(&T);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* C ABI mirroring the reference harness.                                   */

static bf in_bf(const OracleBF* a)
{
    bf x = bf_zero();
    if (!a) return x;
    x.sign = a->sign != 0;
    x.exp = a->exp;
    x.L = (size_t)a->L;
    if (x.L) {
        x.T = (uint32_t*)xmalloc(sizeof(uint32_t) * x.L);
        memcpy(x.T, a->T, sizeof(uint32_t) * x.L);
    }
    return x;
}

static int out_bf(const bf* z, OracleBF* out, uint64_t cap)
{
    out->sign = z->sign;
    out->exp = z->exp;
    out->L = z->L;
    if (z->L > cap) return -1;
    if (z->L) memcpy(out->T, z->T, sizeof(uint32_t) * z->L);
    return 0;
}

int oracle_bf_op(int op, const OracleBF* a, const OracleBF* b, uint64_t p, uint64_t s,
                 OracleBF* out, uint64_t cap)
{
    bf x = in_bf(a), y = in_bf(b), z = bf_zero();
    int rc = 0;
    switch (op) {
    case ORACLE_MUL: z = bf_mul(&x, &y, (size_t)p); break;
    case ORACLE_ADD: z = bf_add(&x, &y, (size_t)p); break;
    case ORACLE_SUB: z = bf_sub(&x, &y, (size_t)p); break;
    case ORACLE_MUL_U32: z = bf_mul_u32(&x, (uint32_t)s); break;
    case ORACLE_RCP: rc = bf_rcp(&x, (size_t)p, &z); break;
    case ORACLE_DIV: { /* div -- BigFloat.cpp:512-515 */
        bf r;
        rc = bf_rcp(&y, (size_t)p, &r);
        if (!rc) {
            z = bf_mul(&x, &r, (size_t)p);
            bf_free(&r);
        }
        break;
    }
    case ORACLE_INVSQRT: rc = bf_invsqrt((uint32_t)s, (size_t)p, &z); break;
    case ORACLE_UCMP: rc = 10 + bf_ucmp(&x, &y); break;
    default: rc = -3;
    }
    if (rc == 0) rc = out_bf(&z, out, cap);
    bf_free(&x);
    bf_free(&y);
    bf_free(&z);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* Chudnovsky binary splitting -- PI.h:64-136                               */

static void bsr(bf* P, bf* Q, bf* R, uint32_t a, uint32_t b, size_t p)
{
    if (b - a == 1) { /* leaf, PI.h:67-88 */
        bf t0 = bf_from_u32(b, 1), c = bf_from_u32(13591409, 1);
        bf t1 = bf_mul_u32(&t0, 545140134);
        bf t2 = bf_add(&t1, &c, 0);
        bf t3 = bf_mul_u32(&t2, 2 * b - 1);
        bf t4 = bf_mul_u32(&t3, 6 * b - 5);
        *P = bf_mul_u32(&t4, 6 * b - 1);
        if (b % 2 == 1) bf_negate(P);
        bf q1 = bf_mul_u32(&t0, b), q2 = bf_mul_u32(&q1, b);
        bf q3 = bf_mul_u32(&q2, 26726400);
        *Q = bf_mul_u32(&q3, 409297880);
        bf r0 = bf_from_u32(2 * b - 1, 1);
        bf r1 = bf_mul_u32(&r0, 6 * b - 5);
        *R = bf_mul_u32(&r1, 6 * b - 1);
        bf_free(&t0); bf_free(&c); bf_free(&t1); bf_free(&t2); bf_free(&t3);
        bf_free(&t4); bf_free(&q1); bf_free(&q2); bf_free(&q3); bf_free(&r0);
        bf_free(&r1);
        return;
    }
    uint32_t m = (a + b) / 2; /* PI.h:90 */
    bf P0, Q0, R0, P1, Q1, R1;
    bsr(&P0, &Q0, &R0, a, m, p);
    bsr(&P1, &Q1, &R1, m, b, p);
    /* P = P0 Q1 + P1 R0 ; Q = Q0 Q1 ; R = R0 R1 -- PI.h:110-112 */
    bf u = bf_mul(&P0, &Q1, p), v = bf_mul(&P1, &R0, p);
    *P = bf_add(&u, &v, p);
    *Q = bf_mul(&Q0, &Q1, p);
    *R = bf_mul(&R0, &R1, p);
    bf_free(&u); bf_free(&v);
    bf_free(&P0); bf_free(&Q0); bf_free(&R0);
    bf_free(&P1); bf_free(&Q1); bf_free(&R1);
}

int oracle_bsr(uint32_t a, uint32_t b, uint64_t p, OracleBF* P, OracleBF* Q, OracleBF* R,
               uint64_t cap)
{
    if (b <= a) return -3;
    bf p_, q_, r_;
    bsr(&p_, &q_, &r_, a, b, (size_t)p);
    int rc = out_bf(&p_, P, cap);
    rc |= out_bf(&q_, Q, cap);
    rc |= out_bf(&r_, R, cap);
    bf_free(&p_);
    bf_free(&q_);
    bf_free(&r_);
    return rc ? -1 : 0;
}

/* Sizes -- PI.h:141-144 */
void oracle_pi_sizes(uint64_t d, uint64_t* hex_digits, uint64_t* p_words, uint64_t* terms)
{
    size_t hex = (size_t)((double)d * log(10) / log(16));
    size_t p = (hex + 9) / 9;
    size_t p_dec = (d + 9) / 9;
    size_t t = (size_t)((double)p_dec * 0.6346230241342037371474889163921741077188431452678) + 1;
    if (hex_digits) *hex_digits = hex;
    if (p_words) *p_words = p;
    if (terms) *terms = t;
}

/* to_string_hex -- BigFloat.cpp:95-106: top word in decimal, '.', then
 * (digits+7)/8 words as %08x, cut to 2 + digits characters. */
static int64_t bf_to_hex(const bf* x, size_t digits, char* buf, uint64_t cap)
{
    size_t nw = (digits + 7) / 8;
    size_t need = 24 + 8 * nw;
    char* s = (char*)xmalloc(need);
    size_t loc = x->L - 1;
    int n = snprintf(s, need, "%u.", x->T[loc]);
    size_t pos = (size_t)n;
    for (size_t i = 0; i < nw; i++) {
        loc--;
        snprintf(s + pos, 9, "%08x", x->T[loc]);
        pos += 8;
    }
    size_t len = 2 + digits < pos ? 2 + digits : pos;
    if (len + 1 > cap) {
        free(s);
        return -1;
    }
    memcpy(buf, s, len);
    buf[len] = 0;
    free(s);
    return (int64_t)len;
}

/* Pi() -- PI.h:138-212 */
int64_t oracle_pi_hex(uint64_t decimal_digits, char* buf, uint64_t cap)
{
    uint64_t hex, p, terms;
    oracle_pi_sizes(decimal_digits, &hex, &p, &terms);
    if ((uint32_t)terms != terms) return -2; /* "Limit Exceeded", PI.h:150-151 */
    bf P, Q, R;
    bsr(&P, &Q, &R, 0, (uint32_t)terms, (size_t)p);
    bf t = bf_mul_u32(&Q, 13591409);
    bf P2 = bf_add(&t, &P, (size_t)p);
    bf Q2 = bf_mul_u32(&Q, 4270934400u);
    bf_free(&t); bf_free(&P); bf_free(&Q); bf_free(&R);
    bf r;
    bf_rcp(&P2, (size_t)p, &r);                 /* div = x * rcp(y), :512-515 */
    bf P3 = bf_mul(&Q2, &r, (size_t)p);
    bf_free(&r); bf_free(&P2); bf_free(&Q2);
    bf Q3;
    bf_invsqrt(10005, (size_t)p, &Q3);
    bf P4 = bf_mul(&P3, &Q3, (size_t)p);
    int64_t n = bf_to_hex(&P4, (size_t)hex, buf, cap);
    bf_free(&P3); bf_free(&Q3); bf_free(&P4);
    return n;
}
