/* Test-infrastructure harness around the UNMODIFIED reference sources.
 *
 * This file is mine; it is compiled together with the reference's own
 * BigFloat.cpp, FFT.cpp and NTT.cpp where they lie (see oracle/Makefile) into
 * oracle/_ref/libpicref.so, the "reference" oracle.  Only tests/, the golden
 * fixture generator and bench.py's CPU-baseline leg load it.  It exposes the
 * reference's BigFloat arithmetic, its NNT transform and its FFT through a
 * plain C ABI so Python tests can compare products, truncation semantics and
 * transform outputs word for word.
 *
 * BigFloat internals (sign/exp/L/T, BigFloat.h:32-36) and NNT internals
 * (p, r, N, W, NTT.cpp:40-42) are private in the reference; the harness opens
 * them with the usual `#define private public` test trick.  Standard headers
 * are included first so the macro only touches the reference's classes. */
#include <stdint.h>
#include <string.h>
#include <string>
#include <memory>
#include <map>
#include <vector>
#include <thread>
#include <future>
#include <sstream>
#include <iomanip>
#include <complex>

#define private public
#include "BigFloat.h"
#include "NTT.cpp"        /* NNT class: NTT.cpp:11-43 (NTT.cpp is not compiled separately) */
#undef private
#include "FFT.h"

extern "C" {

typedef struct {
    int32_t sign;     /* 1 = positive or zero, 0 = negative (BigFloat.h:33) */
    int64_t exp;      /* exponent in 32-bit words (BigFloat.h:34) */
    uint64_t L;       /* number of words (BigFloat.h:35) */
    uint32_t* T;      /* words, little-endian (BigFloat.h:36) */
} RefBF;

static BigFloat to_bf(const RefBF* a)
{
    BigFloat x;
    x.sign = a->sign != 0;
    x.exp = a->exp;
    x.L = (size_t)a->L;
    if (x.L) {
        x.T = std::unique_ptr<uint32_t[]>(new uint32_t[x.L]);
        memcpy(x.T.get(), a->T, sizeof(uint32_t) * x.L);
    }
    return x;
}

/* Copies z into out (capacity cap words).  Returns 0, or -1 when cap is too
 * small (out->L is still set to the needed length). */
static int from_bf(const BigFloat& z, RefBF* out, uint64_t cap)
{
    out->sign = z.sign ? 1 : 0;
    out->exp = z.exp;
    out->L = z.L;
    if (z.L > cap) return -1;
    if (z.L) memcpy(out->T, z.T.get(), sizeof(uint32_t) * z.L);
    return 0;
}

enum {
    REF_MUL = 0,      /* a.mul(b, p, threads)          BigFloat.cpp:326 */
    REF_ADD = 1,      /* a.add(b, p)                   BigFloat.cpp:288 */
    REF_SUB = 2,      /* a.sub(b, p)                   BigFloat.cpp:306 */
    REF_MUL_U32 = 3,  /* a.mul((uint32)s)              BigFloat.cpp:156 */
    REF_RCP = 4,      /* a.rcp(p, threads)             BigFloat.cpp:445 */
    REF_DIV = 5,      /* a.div(b, p, threads)          BigFloat.cpp:512 */
    REF_INVSQRT = 6,  /* invsqrt((uint32)s, p, threads) BigFloat.cpp:516 */
    REF_UCMP = 7      /* a.ucmp(b) -> returned          BigFloat.cpp:123 */
};

/* One reference BigFloat operation.  Returns 0 on success, -1 when the output
 * capacity is too small, -2 when the reference threw, or the ucmp result + 10
 * for REF_UCMP. */
int ref_bf_op(int op, const RefBF* a, const RefBF* b, uint64_t p, uint64_t s,
              int threads, RefBF* out, uint64_t cap)
{
    try {
        BigFloat x = a ? to_bf(a) : BigFloat();
        BigFloat y = b ? to_bf(b) : BigFloat();
        BigFloat z;
        switch (op) {
        case REF_MUL: z = x.mul(y, (size_t)p, threads); break;
        case REF_ADD: z = x.add(y, (size_t)p); break;
        case REF_SUB: z = x.sub(y, (size_t)p); break;
        case REF_MUL_U32: z = x.mul((uint32_t)s); break;
        case REF_RCP: z = x.rcp((size_t)p, threads); break;
        case REF_DIV: z = x.div(y, (size_t)p, threads); break;
        case REF_INVSQRT: z = invsqrt((uint32_t)s, (size_t)p, threads); break;
        case REF_UCMP: return 10 + x.ucmp(y);
        default: return -3;
        }
        return from_bf(z, out, cap);
    } catch (...) {
        return -2;
    }
}

/* to_string_hex (BigFloat.cpp:95-106) of a BigFloat into buf (NUL-terminated). */
int ref_bf_to_hex(const RefBF* a, uint64_t digits, char* buf, uint64_t cap)
{
    std::string s = to_bf(a).to_string_hex((size_t)digits);
    if (s.size() + 1 > cap) return -1;
    memcpy(buf, s.c_str(), s.size() + 1);
    return 0;
}

/* Natural-order NTT of length 2^k with the reference's prime for k
 * (NTT.cpp:125-158), generator (NTT.cpp:104-123) and recursion
 * (NTT.cpp:191-223).  inverse != 0 runs iNTT including the n^-1 scaling
 * (NTT.cpp:80-84).  data is transformed in place.  Reports p, g and the
 * principal root used. */
int ref_nnt(int k, int inverse, uint64_t* data, int threads,
            uint64_t* p_out, uint64_t* g_out, uint64_t* w_out)
{
    if (k < 11 || k > 42) return -1;
    NNT t;
    t.init(1ull << k);
    size_t n = (size_t)1 << k;
    std::vector<uint64_t> dst(n), src(data, data + n);
    if (inverse) t.iNTT(dst.data(), src.data(), threads);
    else t.NTT(dst.data(), src.data(), threads);
    memcpy(data, dst.data(), n * sizeof(uint64_t));
    if (p_out) *p_out = t.p;
    if (g_out) *g_out = t.r;
    if (w_out) *w_out = inverse ? t.iW : t.W;
    return 0;
}

/* The reference's FFT C API (FFT.h) over 2^k interleaved (re, im) doubles. */
int ref_fft(int k, int op, double* data, int threads)
{
    if (k < 1 || k > 26) return -1;
    fft_ensure_table(k);
    __m128d* T = (__m128d*)_mm_malloc(sizeof(__m128d) << k, 64);
    memcpy(T, data, sizeof(__m128d) << k);
    if (op == 0) fft_forward(T, k, threads);
    else fft_inverse(T, k, threads);
    memcpy(data, T, sizeof(__m128d) << k);
    _mm_free(T);
    return 0;
}

/* int_to_fft / fft_to_int (FFT.cpp:485-571) and int_to_ntt / ntt_to_int
 * (NTT.cpp:330-369), for the split and carry layouts. */
int ref_int_to_fft(double* T, int k, const uint32_t* A, uint64_t AL)
{
    try {
        __m128d* buf = (__m128d*)_mm_malloc(sizeof(__m128d) << k, 64);
        int_to_fft(buf, k, A, (size_t)AL);
        memcpy(T, buf, sizeof(__m128d) << k);
        _mm_free(buf);
    } catch (...) { return -2; }
    return 0;
}

int ref_fft_to_int(const double* T, int k, uint32_t* A, uint64_t AL)
{
    try {
        __m128d* buf = (__m128d*)_mm_malloc(sizeof(__m128d) << k, 64);
        memcpy(buf, T, sizeof(__m128d) << k);
        fft_to_int(buf, k, A, (size_t)AL);
        _mm_free(buf);
    } catch (...) { return -2; }
    return 0;
}

int ref_int_to_ntt(uint64_t* T, int k, const uint32_t* A, uint64_t AL)
{
    try { int_to_ntt(T, k, A, (size_t)AL); } catch (...) { return -2; }
    return 0;
}

int ref_ntt_to_int(uint64_t* T, int k, uint32_t* A, uint64_t AL)
{
    try { ntt_to_int(T, k, A, (size_t)AL); } catch (...) { return -2; }
    return 0;
}

}  /* extern "C" */
