// Exact products: piece split, multi-prime NTT convolution, CRT and carry.
#include <math.h>
#include <string.h>

#include <atomic>
#include <utility>

#include "carry.cuh"
#include "common.cuh"
#include "fp64mod.cuh"
#include "mul.cuh"

namespace pic {

static inline int ceil_log2(size_t n)
{
    int k = 0;
    while (((size_t)1 << k) < n) k++;
    return k;
}

// ---- split -----------------------------------------------------------------
// Three-prime form: piece j = a[2j] | a[2j+1] << 32, reduced mod each prime.
__global__ void split3_kernel(uint64_t* __restrict__ out, const uint32_t* __restrict__ a, size_t na, size_t N,
                              uint64_t p0, uint64_t p1, uint64_t p2)
{
    const size_t np = (na + 1) / 2;
    for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < N; j += (size_t)gridDim.x * blockDim.x) {
        uint64_t v = 0;
        if (j < np) {
            const uint64_t lo = a[2 * j];
            const uint64_t hi = (2 * j + 1 < na) ? a[2 * j + 1] : 0u;
            v = lo | (hi << 32);
        }
        out[j] = piece_to_strict(v, p0);
        out[N + j] = piece_to_strict(v, p1);
        out[2 * N + j] = piece_to_strict(v, p2);
    }
}

// Pieces first .. first + 2^k - 1 of a (zero past its end) -> residues at
// out + q * stride.
__global__ void split3_off_kernel(uint64_t* __restrict__ out, size_t stride, const uint32_t* __restrict__ a,
                                  size_t na, size_t first, size_t N, uint64_t p0, uint64_t p1, uint64_t p2)
{
    for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < N; j += (size_t)gridDim.x * blockDim.x) {
        const size_t wi = 2 * (first + j);
        uint64_t v = 0;
        if (wi < na) {
            v = a[wi];
            if (wi + 1 < na) v |= (uint64_t)a[wi + 1] << 32;
        }
        out[j] = piece_to_strict(v, p0);
        out[stride + j] = piece_to_strict(v, p1);
        out[2 * stride + j] = piece_to_strict(v, p2);
    }
}

// Reference layout, int_to_ntt NTT.cpp:330-341: two 16-bit points per word.
__global__ void split16_kernel(uint64_t* __restrict__ T, size_t N, const uint32_t* __restrict__ A, size_t AL)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        const size_t w = i >> 1;
        uint64_t v = 0;
        if (w < AL) v = (i & 1) ? (A[w] >> 16) : (A[w] & 0xffffu);
        T[i] = v;
    }
}

// ---- coefficient -> word conversion ----------------------------------------
constexpr int kCvtThreads = 256;
constexpr int kCvtLPT = 2;  // 64-bit limbs per thread
constexpr size_t kCvtLPC = (size_t)kCvtThreads * kCvtLPT;
constexpr size_t kCvtWPC = 2 * kCvtLPC;
// The CRT conversion needs three coefficients below its first limb, so a CTA
// of 256 threads computes 512 coefficients (two per thread, no thread a
// third) and owns the 509 limbs they complete.
constexpr size_t kCrtSlots = (size_t)kCvtThreads * kCvtLPT;
constexpr size_t kCrtLPC = kCrtSlots - 3;
constexpr size_t kCrtWPC = 2 * kCrtLPC;

struct Crt3Consts {
    uint64_t p[3];
    uint32_t c[3];      // p = c 2^32 + 1
    ulonglong2 scale[3];  // N^-1 R^depth mod p_q (Shoup pair): undoes the pointwise R^-1 and the unscaled inverse
    ulonglong2 inv01;     // p0^-1 mod p1
    ulonglong2 p0m2;      // p0 mod p2
    ulonglong2 inv012;    // (p0 p1)^-1 mod p2
    uint64_t p0p1_lo, p0p1_hi;
    uint64_t off[3];      // 2^159 mod p_q when every coefficient gets the offset 2^159, else 0
};

// x * w mod p in [0, p) for a Shoup pair w (product primes c 2^32 + 1).
__device__ __forceinline__ uint64_t crt_mul(uint64_t x, const ulonglong2& w, uint64_t p, uint32_t c)
{
    const uint64_t r = shoup_lazy32(x, w.x, w.y, c);
    return r >= p ? r - p : r;
}

// Garner's CRT: x = r0 + p0 (v1 + p1 v2), 0 <= x < p0 p1 p2, as three limbs.
// Inputs may be any 64-bit residue representatives (lazy transforms).  With
// the offset set, x is the coefficient plus 2^159 (signed coefficients of
// magnitude below 2^159 come out nonnegative and exact).
__device__ __forceinline__ void crt3(const Crt3Consts& C, uint64_t y0, uint64_t y1, uint64_t y2, uint64_t& l0,
                                     uint64_t& l1, uint64_t& l2)
{
    const uint64_t r0s = crt_mul(y0, C.scale[0], C.p[0], C.c[0]);
    const uint64_t r1s = crt_mul(y1, C.scale[1], C.p[1], C.c[1]);
    const uint64_t r2o = crt_mul(y2, C.scale[2], C.p[2], C.c[2]);
    const uint64_t r0 = add_mod(r0s, C.off[0], C.p[0]);
    const uint64_t r1 = add_mod(r1s, C.off[1], C.p[1]);
    const uint64_t r2 = add_mod(r2o, C.off[2], C.p[2]);
    const uint64_t r0m1 = r0 >= C.p[1] ? r0 - C.p[1] : r0;
    const uint64_t v1 = crt_mul(sub_mod(r1, r0m1, C.p[1]), C.inv01, C.p[1], C.c[1]);
    const uint64_t r0m2 = r0 >= C.p[2] ? r0 - C.p[2] : r0;
    uint64_t t = sub_mod(r2, r0m2, C.p[2]);
    t = sub_mod(t, crt_mul(v1, C.p0m2, C.p[2], C.c[2]), C.p[2]);
    const uint64_t v2 = crt_mul(t, C.inv012, C.p[2], C.c[2]);
    // p0 * v1 + r0 = v1 + (c0 v1) 2^32 + r0 with two 32 x 32 products
    const uint64_t x = (uint64_t)C.c[0] * (uint32_t)v1, y = (uint64_t)C.c[0] * (uint32_t)(v1 >> 32);
    uint64_t a0 = v1 + (x << 32), a1 = (x >> 32) + y + (a0 < v1);
    a0 += r0;
    a1 += (a0 < r0);
    // (p0 p1) * v2
    const uint64_t b0 = C.p0p1_lo * v2;
    uint64_t b1 = mulhi64(C.p0p1_lo, v2);
    const uint64_t t1 = C.p0p1_hi * v2;
    uint64_t b2 = mulhi64(C.p0p1_hi, v2);
    b1 += t1;
    b2 += (b1 < t1);
    l0 = a0 + b0;
    const uint64_t c0 = l0 < b0;
    uint64_t s1 = a1 + b1;
    uint64_t c1 = s1 < b1;
    s1 += c0;
    c1 += (s1 < c0);
    l1 = s1;
    l2 = b2 + c1;
}

// Shared tail of both conversions: limb digits (T = D_i + C_(i-1)) -> words
// with in-block carry resolution; writes the CTA's (G, P).
template <int NL>
__device__ __forceinline__ void limbs_to_words(const uint64_t (&dig)[NL], const uint32_t (&gen)[NL],
                                               size_t first_limb, uint32_t* z, size_t zw, uint32_t* agg_slot)
{
    uint32_t gp = kGPIdentity;
#pragma unroll
    for (int u = 0; u < NL; u++) {
        const size_t w = 2 * (first_limb + u);
        const uint32_t lo = (uint32_t)dig[u], hi = (uint32_t)(dig[u] >> 32);
        if (w < zw) gp = gp_combine(gp, (uint32_t)(lo == 0xffffffffu) << 1);
        if (w + 1 < zw) gp = gp_combine(gp, gen[u] | ((uint32_t)(hi == 0xffffffffu) << 1));
    }
    uint32_t total;
    uint32_t cin = block_gp_scan(gp, &total) & 1u;
#pragma unroll
    for (int u = 0; u < NL; u++) {
        const size_t w = 2 * (first_limb + u);
        const uint32_t lo = (uint32_t)dig[u], hi = (uint32_t)(dig[u] >> 32);
        if (w < zw) z[w] = lo + cin;
        cin = (uint32_t)(lo == 0xffffffffu) & cin;
        if (w + 1 < zw) z[w + 1] = hi + cin;
        cin = gen[u] | ((uint32_t)(hi == 0xffffffffu) & cin);
    }
    if (threadIdx.x == 0) *agg_slot = total;
}

__device__ __forceinline__ void add128(uint64_t& lo, uint64_t& hi, uint64_t v)
{
    lo += v;
    hi += (lo < v);
}

// Three-prime residues y[q * pstride + j] -> words.  Limb i (64 bits)
// collects x_i.l0 + x_(i-1).l1 + x_(i-2).l2 (< 3 * 2^64).  One CTA handles
// limbs [i0, i0 + kCrtLPC) of one product; slot t of xs holds coefficient
// i0 - 3 + t.
__device__ __forceinline__ void crt3_block(const uint64_t* __restrict__ Y, size_t pstride, size_t ncoef,
                                           const Crt3Consts& C, uint32_t* __restrict__ z, size_t zw, int64_t i0,
                                           uint32_t* agg_slot)
{
    __shared__ uint64_t xs[kCrtSlots * 3];
    const int64_t climit = (int64_t)((zw + 1) / 2);  // limbs this product needs
    for (int t = threadIdx.x; t < (int)kCrtSlots; t += blockDim.x) {
        const int64_t j = i0 - 3 + t;
        uint64_t l0 = 0, l1 = 0, l2 = 0;
        if (j >= 0 && (size_t)j < ncoef && j < climit)
            crt3(C, Y[j], Y[pstride + j], Y[2 * pstride + j], l0, l1, l2);
        xs[3 * t] = l0;
        xs[3 * t + 1] = l1;
        xs[3 * t + 2] = l2;
    }
    __syncthreads();
    uint64_t dig[kCvtLPT];
    uint32_t gen[kCvtLPT];
#pragma unroll
    for (int u = 0; u < kCvtLPT; u++) {
        const int l = threadIdx.x * kCvtLPT + u;  // limb i0 + l, xs slot l + 3
        dig[u] = 0;
        gen[u] = 0;
        if (l < (int)kCrtLPC) {
            const int li = l + 3;
            uint64_t slo = xs[3 * li], shi = 0;
            add128(slo, shi, xs[3 * (li - 1) + 1]);
            add128(slo, shi, xs[3 * (li - 2) + 2]);
            uint64_t plo = xs[3 * (li - 1)], phi = 0;
            add128(plo, phi, xs[3 * (li - 2) + 1]);
            add128(plo, phi, xs[3 * (li - 3) + 2]);
            const uint64_t d = slo + phi;
            dig[u] = d;
            gen[u] = d < slo;
        }
    }
    // words past this CTA's limbs belong to the next CTA
    const size_t zend = 2 * ((size_t)i0 + kCrtLPC);
    limbs_to_words(dig, gen, (size_t)i0 + threadIdx.x * kCvtLPT, z, zw < zend ? zw : zend, agg_slot);
}

__global__ void __launch_bounds__(kCvtThreads) crt3_k1(const uint64_t* __restrict__ Y, size_t N, size_t ncoef,
                                                       Crt3Consts C, uint32_t* __restrict__ z, size_t zw,
                                                       uint32_t* agg)
{
    crt3_block(Y, N, ncoef, C, z, zw, (int64_t)blockIdx.x * (int64_t)kCrtLPC, agg + blockIdx.x);
}

// Batched: product i has residues at Y + i * istride (+ q * pstride), zlen[i]
// words out at z + i * zcap; cpp CTAs per product.
__global__ void __launch_bounds__(kCvtThreads) crt3_batch_k1(const uint64_t* __restrict__ Y, size_t istride,
                                                             size_t pstride, size_t ncoef, Crt3Consts C,
                                                             uint32_t* __restrict__ z, uint32_t zcap,
                                                             const uint32_t* __restrict__ zlen, size_t cpp,
                                                             uint32_t* agg)
{
    const size_t prod = blockIdx.x / cpp, lc = blockIdx.x % cpp;
    crt3_block(Y + prod * istride, pstride, ncoef, C, z + prod * (size_t)zcap, zlen[prod],
               (int64_t)lc * (int64_t)kCrtLPC, agg + blockIdx.x);
}

// Coefficients c_j at bit offsets bits * j (8 <= bits <= 16) -> words.  Limb
// i (bits [64i, 64i+64)) collects lo64(c_j << r_j) for the j with
// floor(bits j / 64) == i and hi64(c_j << r_j) for those with i - 1, where
// r_j = bits j mod 64.  A loader supplies c_j (< 2^64).
constexpr int kStageMax = (int)(64 * (kCvtLPC + 2) / 8 + 2);

__device__ __forceinline__ int64_t first_coef(int64_t limb, int bits)
{
    return limb <= 0 ? 0 : (64 * limb + bits - 1) / bits;
}

__device__ __forceinline__ void limb_sum(const uint64_t* cs, int64_t jlo, int64_t limb, int bits, uint64_t& lo,
                                         uint64_t& hi)
{
    lo = 0;
    hi = 0;
    if (limb < 0) return;
    const int64_t a = first_coef(limb - 1, bits), b = first_coef(limb, bits), c = first_coef(limb + 1, bits);
    if (limb >= 1)
        for (int64_t j = a; j < b; j++) {
            const int r = (int)((bits * j) & 63);
            if (r) add128(lo, hi, cs[j - jlo] >> (64 - r));
        }
    for (int64_t j = b; j < c; j++) add128(lo, hi, cs[j - jlo] << ((bits * j) & 63));
}

struct NttCoefLoader {
    const uint64_t* c;
    uint64_t scale, p, pinv;
    __device__ __forceinline__ uint64_t operator()(size_t j, double&) const
    {
        uint64_t v = c[j];
        return scale ? mont_mul(v, scale, p, pinv) : v;
    }
};

struct FftCoefLoader {
    const double2* T;
    double scale;
    __device__ __forceinline__ uint64_t operator()(size_t j, double& emax) const
    {
        const double f = T[j].x * scale;
        const double r = rint(f);
        const double e = fabs(f - r);
        if (e > emax) emax = e;
        return r > 0 ? (uint64_t)r : 0;
    }
};

template <class Loader>
__global__ void __launch_bounds__(kCvtThreads) coefbits_k1(Loader ld, size_t ncoef, int bits,
                                                           uint32_t* __restrict__ z, size_t zw, uint32_t* agg,
                                                           unsigned long long* err_bits)
{
    __shared__ uint64_t cs[kStageMax];
    const int64_t i0 = (int64_t)blockIdx.x * (int64_t)kCvtLPC;
    const int64_t jlo = first_coef(i0 - 2, bits), jhi = first_coef(i0 + (int64_t)kCvtLPC, bits);
    double emax = 0.0;
    for (int64_t t = threadIdx.x; t < jhi - jlo; t += blockDim.x) {
        const int64_t j = jlo + t;
        cs[t] = (j < (int64_t)ncoef) ? ld((size_t)j, emax) : 0;
    }
    if (err_bits) {
#pragma unroll
        for (int off = 16; off; off >>= 1) emax = fmax(emax, __shfl_xor_sync(0xffffffffu, emax, off));
        if ((threadIdx.x & 31) == 0 && emax > 0.0) atomicMax(err_bits, (unsigned long long)__double_as_longlong(emax));
    }
    __syncthreads();
    uint64_t dig[kCvtLPT];
    uint32_t gen[kCvtLPT];
#pragma unroll
    for (int u = 0; u < kCvtLPT; u++) {
        const int64_t i = i0 + threadIdx.x * kCvtLPT + u;
        uint64_t slo, shi, plo, phi;
        limb_sum(cs, jlo, i, bits, slo, shi);
        limb_sum(cs, jlo, i - 1, bits, plo, phi);
        const uint64_t d = slo + phi;
        dig[u] = d;
        gen[u] = d < slo;
    }
    limbs_to_words(dig, gen, (size_t)i0 + threadIdx.x * kCvtLPT, z, zw, agg + blockIdx.x);
}

// Carries between the CTAs of a coefficient-bits conversion (kCvtLPC limbs
// per CTA; the CRT conversions own kCrtLPC and ripple with kCrtWPC).
static void finish_scan(uint32_t* z, size_t zw, uint32_t* agg, size_t nctas, cudaStream_t s)
{
    carry_scan_aggregates(agg, nctas, nullptr, s);
    carry_ripple(z, zw, kCvtWPC, agg, nctas, kCarryAdd, s);
}

void coef16_to_words(const uint64_t* c, size_t ncoef, uint64_t scale_mont, uint64_t p, uint64_t pinv_neg,
                     uint32_t* z, size_t zw, cudaStream_t s)
{
    if (zw == 0) return;
    const size_t nlimbs = (zw + 1) / 2;
    const size_t nctas = (nlimbs + kCvtLPC - 1) / kCvtLPC;
    DevBuf<uint32_t> agg(nctas, s);
    ProfScope ps(KC_CRT, 8.0 * (double)ncoef + 4.0 * (double)zw, s);
    coefbits_k1<NttCoefLoader><<<(unsigned)nctas, kCvtThreads, 0, s>>>(
        NttCoefLoader{c, scale_mont, p, pinv_neg}, ncoef, 16, z, zw, agg.get(), nullptr);
    PIC_CHECK_LAUNCH();
    count_launch();
    finish_scan(z, zw, agg.get(), nctas, s);
}

double fft_coef_to_words(const double2* T, size_t ncoef, double scale, int bits, uint32_t* z, size_t zw,
                         cudaStream_t s)
{
    PIC_REQUIRE(bits >= 8 && bits <= 16, PIC_ERR_INVALID, "FFT piece width out of range");
    if (zw == 0) return 0.0;
    const size_t nlimbs = (zw + 1) / 2;
    const size_t nctas = (nlimbs + kCvtLPC - 1) / kCvtLPC;
    DevBuf<uint32_t> agg(nctas, s);
    DevBuf<unsigned long long> err(1, s);
    PIC_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(unsigned long long), s));
    ProfScope ps(KC_CRT, 16.0 * (double)ncoef + 4.0 * (double)zw, s);
    coefbits_k1<FftCoefLoader><<<(unsigned)nctas, kCvtThreads, 0, s>>>(FftCoefLoader{T, scale}, ncoef, bits, z,
                                                                        zw, agg.get(), err.get());
    PIC_CHECK_LAUNCH();
    count_launch();
    finish_scan(z, zw, agg.get(), nctas, s);
    unsigned long long eb = 0;
    read_words((uint32_t*)&eb, (const uint32_t*)err.get(), 2, s);
    double e;
    memcpy(&e, &eb, sizeof e);
    return e;
}

// Scale folded into the CRT: multiplying by R^depth N^-1 undoes `depth`
// pointwise Montgomery products (each contributes R^-1) and the unscaled
// inverse (N).  Every constant is a Shoup pair (value, companion).
static Crt3Consts make_crt3(int k, int depth)
{
    Crt3Consts C;
    const uint64_t N = (uint64_t)1 << k;
    auto pair = [](uint64_t w, uint64_t p) { return make_ulonglong2(w, shoup_companion(w, p)); };
    for (int q = 0; q < 3; q++) {
        const uint64_t p = kProductPrimes[q];
        C.p[q] = p;
        C.c[q] = (uint32_t)(p >> 32);
        uint64_t sc = host_powmod(N % p, p - 2, p);
        for (int d = 0; d < depth; d++) sc = to_mont(sc, p);
        C.scale[q] = pair(sc, p);  // y * N^-1 R^depth
    }
    const uint64_t p0 = C.p[0], p1 = C.p[1], p2 = C.p[2];
    C.inv01 = pair(host_powmod(p0 % p1, p1 - 2, p1), p1);
    C.p0m2 = pair(p0 % p2, p2);
    const uint64_t p01m2 = host_mulmod(p0 % p2, p1 % p2, p2);
    C.inv012 = pair(host_powmod(p01m2, p2 - 2, p2), p2);
    const unsigned __int128 p01 = (unsigned __int128)p0 * p1;
    C.p0p1_lo = (uint64_t)p01;
    C.p0p1_hi = (uint64_t)(p01 >> 64);
    for (int q = 0; q < 3; q++) C.off[q] = 0;
    return C;
}

static NttBatch ntt3_batch(uint64_t* data, int k)
{
    NttBatch bat;
    bat.data = data;
    bat.stride = (size_t)1 << k;
    bat.count = 3;
    bat.per_prime = 1;
    for (int q = 0; q < 3; q++) bat.prime[q] = prime_tables(kProductPrimes[q]).dev;
    return bat;
}

void ntt3_forward_operand(uint64_t* out, int k, const uint32_t* a, size_t na, cudaStream_t s)
{
    const size_t N = (size_t)1 << k;
    {
        ProfScope ps(KC_SPLIT, 4.0 * (double)na + 24.0 * (double)N, s);
        split3_kernel<<<grid_for(N, 256), 256, 0, s>>>(out, a, na, N, kProductPrimes[0], kProductPrimes[1],
                                                       kProductPrimes[2]);
        PIC_CHECK_LAUNCH();
        count_launch();
    }
    ntt_forward_dif(ntt3_batch(out, k), k, s);
}

void ntt3_pointwise(uint64_t* a, const uint64_t* b, int k, cudaStream_t s)
{
    ntt_pointwise_mont(ntt3_batch(a, k), b, k, s);
}

void ntt3_inverse_to_words(uint64_t* y, int k, size_t ncoef, int depth, uint32_t* z, size_t zw, cudaStream_t s)
{
    ntt_inverse_dit(ntt3_batch(y, k), k, s);
    const Crt3Consts C = make_crt3(k, depth);
    const size_t nlimbs = (zw + 1) / 2;
    const size_t nctas = (nlimbs + kCrtLPC - 1) / kCrtLPC;
    DevBuf<uint32_t> agg(nctas, s);
    ProfScope ps(KC_CRT, 24.0 * (double)ncoef + 4.0 * (double)zw, s);
    crt3_k1<<<(unsigned)nctas, kCvtThreads, 0, s>>>(y, (size_t)1 << k, ncoef, C, z, zw, agg.get());
    PIC_CHECK_LAUNCH();
    count_launch();
    carry_scan_aggregates(agg.get(), nctas, nullptr, s);
    carry_ripple(z, zw, kCrtWPC, agg.get(), nctas, kCarryAdd, s);
}

void ntt3_batch_to_words(const uint64_t* y, size_t istride, size_t pstride, size_t count, int k, uint32_t* z,
                         uint32_t zcap, const uint32_t* zlen, cudaStream_t s, size_t ncoef, bool offset)
{
    if (count == 0) return;
    if (ncoef == 0) ncoef = (size_t)1 << k;
    Crt3Consts C = make_crt3(k, 1);
    if (offset)
        for (int q = 0; q < 3; q++) C.off[q] = host_powmod(2, 159, C.p[q]);
    const size_t cpp = (((size_t)zcap + 1) / 2 + kCrtLPC - 1) / kCrtLPC;
    const size_t nctas = count * cpp;
    DevBuf<uint32_t> agg(nctas, s);
    {
        ProfScope ps(KC_CRT, (24.0 * (double)ncoef + 4.0 * zcap) * (double)count, s);
        crt3_batch_k1<<<(unsigned)nctas, kCvtThreads, 0, s>>>(y, istride, pstride, ncoef, C, z, zcap, zlen,
                                                              cpp, agg.get());
        PIC_CHECK_LAUNCH();
        count_launch();
    }
    carry_scan_segments(agg.get(), count, cpp, s);
    carry_ripple_batch(z, zcap, zlen, kCrtWPC, agg.get(), count, cpp, s);
}

// Pieces used by the allocation-free product (noalloc.cu): the same split and
// CRT + carry kernels, with every buffer supplied by the caller.
void split3_into(uint64_t* out, int k, const uint32_t* a, size_t na, const uint64_t primes[3], cudaStream_t s)
{
    const size_t N = (size_t)1 << k;
    split3_kernel<<<grid_for(N, 256), 256, 0, s>>>(out, a, na, N, primes[0], primes[1], primes[2]);
    PIC_CHECK_LAUNCH();
    count_launch();
}

size_t crt3_scratch_ctas(size_t zw) { return ((zw + 1) / 2 + kCrtLPC - 1) / kCrtLPC; }

void crt3_to_words_scratch(const uint64_t* y, int k, size_t ncoef, uint32_t* z, size_t zw, uint32_t* agg,
                           cudaStream_t s)
{
    const Crt3Consts C = make_crt3(k, 1);
    const size_t nctas = crt3_scratch_ctas(zw);
    crt3_k1<<<(unsigned)nctas, kCvtThreads, 0, s>>>(y, (size_t)1 << k, ncoef, C, z, zw, agg);
    PIC_CHECK_LAUNCH();
    count_launch();
    carry_scan_aggregates(agg, nctas, nullptr, s);
    carry_ripple(z, zw, kCrtWPC, agg, nctas, kCarryAdd, s);
}

// Wrapped products.  A product of operands of sa and sb pieces has
// L = sa + sb - 1 coefficients c_0..c_(L-1).  When L exceeds the main
// transform length Nm (but sa, sb <= Nm), the cyclic product of length Nm
// holds c_j + c_(Nm+j) for j < W = L - Nm.  The W top coefficients depend only
// on the top W pieces of each operand (a from index Nm - sb + 1, b from
// Nm - sa + 1): the product of those pieces, d, gives c_(Nm+j) = d_(W-1+j),
// and its cyclic length T >= 2W - 1 keeps those indices free of wrap.  For
// each of the W positions:
//   y[j] <- y[j] - h (kept nonnegative by adding p), y[Nm + j] <- h
// (inverse outputs arrive in [0, 8p) and are first brought below 4p),
// with h = d_(W-1+j) * Nm / T so that both halves carry the same scale Nm.
// y items have stride ystride >= Nm + W; tail items have stride T.  `item`
// selects which children hold products (all for P, the even ones for Q, R).
__global__ void wrap_fix_kernel(uint64_t* __restrict__ y, size_t ystride, const uint64_t* __restrict__ tail,
                                size_t T, size_t nitems, size_t item_mul, size_t nchild, size_t Nm, size_t W,
                                Mod64 m0, Mod64 m1, Mod64 m2, uint64_t c0, uint64_t c1, uint64_t c2)
{
    const size_t total = 3 * nitems * W;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < total; g += (size_t)gridDim.x * blockDim.x) {
        const size_t q = g / (nitems * W);
        const size_t r = g - q * nitems * W;
        const size_t it = r / W, j = r - it * W;
        const Mod64& M = q == 0 ? m0 : (q == 1 ? m1 : m2);
        const uint64_t cT = q == 0 ? c0 : (q == 1 ? c1 : c2);
        const size_t child = q * nchild + it * item_mul;
        const uint64_t h = mont_mul(tail[child * T + W - 1 + j], cT, M);  // < p
        uint64_t* yi = y + child * ystride;
        const uint64_t p4 = 4 * M.p;
        uint64_t v = yi[j];  // lazy inverse output, < 8p
        v = v >= p4 ? v - p4 : v;
        yi[j] = v + M.p - h;  // < 5p < 2^64: the CRT reduces any 64-bit input
        yi[Nm + j] = h;
    }
}

void launch_wrap_fix(uint64_t* y, size_t ystride, const uint64_t* tail, size_t T, size_t nitems, size_t item_mul,
                     size_t nchild, size_t Nm, size_t W, const uint64_t cT[3], cudaStream_t s)
{
    const Mod64 m0 = make_mod(kProductPrimes[0]), m1 = make_mod(kProductPrimes[1]), m2 = make_mod(kProductPrimes[2]);
    wrap_fix_kernel<<<grid_for(3 * nitems * W, 256), 256, 0, s>>>(y, ystride, tail, T, nitems, item_mul, nchild, Nm,
                                                                W, m0, m1, m2, cT[0], cT[1], cT[2]);
    PIC_CHECK_LAUNCH();
}

// ---- products ----------------------------------------------------------------
static bool g_mul_wrap = true;
void mul_set_wrap(bool on) { g_mul_wrap = on; }
bool mul_wrap() { return g_mul_wrap; }

static NttBatch ntt3_batch_stride(uint64_t* data, size_t stride)
{
    NttBatch bat;
    bat.data = data;
    bat.stride = stride;
    bat.count = 3;
    bat.per_prime = 1;
    for (int q = 0; q < 3; q++) bat.prime[q] = prime_tables(kProductPrimes[q]).dev;
    return bat;
}

// ---- a held forward transform (transform reuse in the Newton steps) ----------
// While an OperandHold for (src, n) is alive on this thread, three-prime
// products that take that operand reuse its forward transform at main length
// 2^k instead of transforming it again: the first such product computes it
// (split + forward, stride 2^k) and keeps it, later ones read it.  The plain
// product at 2^k and the main part of a wrapped product at Nm = 2^k split the
// operand the same way (pieces 0 .. 2^k - 1, zero above), so one transform
// serves both.  Only the operand's words, length and k decide a match.
namespace {
struct HeldOperand {
    const uint32_t* src = nullptr;
    size_t n = 0;
    int k = -1;
    int form = kFormInt;
    DevBuf<uint64_t> T;  // 3 x 2^k residues, transforms 2^k apart, bit-reversed order
};
thread_local HeldOperand* t_held = nullptr;
std::atomic<uint64_t> g_held_reuses{0};
}  // namespace

OperandHold::OperandHold(const uint32_t* src, size_t n) : prev_(t_held)
{
    auto* h = new HeldOperand;
    h->src = src;
    h->n = n;
    held_ = h;
    t_held = h;
}

OperandHold::~OperandHold()
{
    t_held = static_cast<HeldOperand*>(prev_);
    delete static_cast<HeldOperand*>(held_);
}

uint64_t held_transform_reuses() { return g_held_reuses.load(); }

static bool is_held(const uint32_t* x, size_t n) { return t_held && t_held->src == x && t_held->n == n; }

void ntt3d_forward_operand(uint64_t* out, int k, const uint32_t* a, size_t na, cudaStream_t s);

// The held operand's forward transform at length 2^k (stride 2^k) in the
// given product form, computed on first use at that length and form.
static const uint64_t* held_transform(int k, int form, cudaStream_t s)
{
    HeldOperand* h = t_held;
    if (h->k != k || h->form != form) {
        h->T = DevBuf<uint64_t>(3 * ((size_t)1 << k), s);
        if (form == kFormDbl) ntt3d_forward_operand(h->T.get(), k, h->src, h->n, s);
        else ntt3_forward_operand(h->T.get(), k, h->src, h->n, s);
        h->k = k;
        h->form = form;
    } else {
        g_held_reuses.fetch_add(1);
    }
    return h->T.get();
}

// Copies three transforms of 2^k residues from stride `from` to stride `to`.
static void copy_transforms(uint64_t* dst, size_t to, const uint64_t* src, size_t from, int k, cudaStream_t s)
{
    PIC_CUDA(cudaMemcpy2DAsync(dst, to * sizeof(uint64_t), src, from * sizeof(uint64_t),
                               sizeof(uint64_t) << k, 3, cudaMemcpyDeviceToDevice, s));
}

// The wrapped form of mul_ntt3 (see wrap_fix_kernel): main transforms of
// length Nm = 2^km, tails of length 2^kt over the top W pieces.
static void mul_ntt3_wrapped(uint32_t* z, const uint32_t* a, size_t na, const uint32_t* b, size_t nb, int km,
                             int kt, cudaStream_t s)
{
    const size_t zw = na + nb;
    const size_t pa = (na + 1) / 2, pb = (nb + 1) / 2;
    const size_t L = pa + pb - 1;
    const size_t Nm = (size_t)1 << km, T = (size_t)1 << kt, W = L - Nm;
    const size_t ST = Nm + ((W + 15) & ~(size_t)15);
    const bool square = (a == b && na == nb);
    const uint64_t P0 = kProductPrimes[0], P1 = kProductPrimes[1], P2 = kProductPrimes[2];
    // a held b (or a held square) brings its main transform with it
    const uint64_t* held = is_held(b, nb) ? held_transform(km, kFormInt, s) : nullptr;
    DevBuf<uint64_t> A(3 * ST, s), B(square || held ? 0 : 3 * ST, s), tA(3 * T, s), tB(square ? 0 : 3 * T, s);
    {
        ProfScope ps(KC_SPLIT, 4.0 * (double)(na + nb) + 24.0 * (double)(2 * (Nm + T)), s);
        if (!(held && square))
            split3_off_kernel<<<grid_for(Nm, 256), 256, 0, s>>>(A.get(), ST, a, na, 0, Nm, P0, P1, P2);
        split3_off_kernel<<<grid_for(T, 256), 256, 0, s>>>(tA.get(), T, a, na, Nm - pb + 1, T, P0, P1, P2);
        if (!square) {
            if (!held)
                split3_off_kernel<<<grid_for(Nm, 256), 256, 0, s>>>(B.get(), ST, b, nb, 0, Nm, P0, P1, P2);
            split3_off_kernel<<<grid_for(T, 256), 256, 0, s>>>(tB.get(), T, b, nb, Nm - pa + 1, T, P0, P1, P2);
        }
        PIC_CHECK_LAUNCH();
        count_launch((held && square ? 0 : 1) + 1 + (square ? 0 : (held ? 1 : 2)));
    }
    const NttBatch mA = ntt3_batch_stride(A.get(), ST), mB = ntt3_batch_stride(B.get(), ST);
    const NttBatch xA = ntt3_batch_stride(tA.get(), T), xB = ntt3_batch_stride(tB.get(), T);
    if (held && square) copy_transforms(A.get(), ST, held, Nm, km, s);
    else ntt_forward_dif(mA, km, s);
    ntt_forward_dif(xA, kt, s);
    if (!square) {
        if (!held) ntt_forward_dif(mB, km, s);
        ntt_forward_dif(xB, kt, s);
    }
    if (held) ntt_pointwise_mont(mA, held, km, s, Nm);
    else ntt_pointwise_mont(mA, square ? A.get() : B.get(), km, s);
    ntt_pointwise_mont(xA, square ? tA.get() : tB.get(), kt, s);
    ntt_inverse_dit(mA, km, s);
    ntt_inverse_dit(xA, kt, s);
    uint64_t cT[3];
    for (int q = 0; q < 3; q++) cT[q] = to_mont((uint64_t)(Nm / T), kProductPrimes[q]);
    {
        ProfScope ps(KC_NTT_POINTWISE, 3.0 * (double)W * 24.0, s);
        launch_wrap_fix(A.get(), ST, tA.get(), T, 1, 1, 1, Nm, W, cT, s);
        count_launch();
    }
    const Crt3Consts C = make_crt3(km, 1);
    const size_t nctas = crt3_scratch_ctas(zw);
    DevBuf<uint32_t> agg(nctas, s);
    ProfScope ps(KC_CRT, 24.0 * (double)L + 4.0 * (double)zw, s);
    crt3_k1<<<(unsigned)nctas, kCvtThreads, 0, s>>>(A.get(), ST, L, C, z, zw, agg.get());
    PIC_CHECK_LAUNCH();
    count_launch();
    carry_scan_aggregates(agg.get(), nctas, nullptr, s);
    carry_ripple(z, zw, kCrtWPC, agg.get(), nctas, kCarryAdd, s);
}

void mul_ntt3(uint32_t* z, const uint32_t* a, size_t na, const uint32_t* b, size_t nb, cudaStream_t s)
{
    if (is_held(a, na) && !(a == b && na == nb)) {  // the held operand goes second
        std::swap(a, b);
        std::swap(na, nb);
    }
    const size_t zw = na + nb;
    const size_t pa = (na + 1) / 2, pb = (nb + 1) / 2;
    const size_t ncoef = pa + pb - 1;
    int k = ceil_log2(ncoef);
    if (k < 1) k = 1;
    PIC_REQUIRE(k <= 30, PIC_ERR_LENGTH, "product too long for the three-prime NTT (2^30 points)");
    const size_t N = (size_t)1 << k;
    if (g_mul_wrap && k >= 4) {
        // wrapped when the product just exceeds a power of two and the tail is short
        const size_t Nm = N / 2;
        if (std::max(pa, pb) <= Nm && ncoef > Nm) {
            const size_t W = ncoef - Nm;
            int kt = ceil_log2(2 * W - 1);
            if (kt < 2) kt = 2;
            if (((size_t)1 << kt) <= Nm / 2) {
                mul_ntt3_wrapped(z, a, na, b, nb, k - 1, kt, s);
                return;
            }
        }
    }
    const bool square = (a == b && na == nb);
    const uint64_t* held = is_held(b, nb) ? held_transform(k, kFormInt, s) : nullptr;
    DevBuf<uint64_t> A(3 * N, s);
    DevBuf<uint64_t> B(square || held ? 0 : 3 * N, s);
    if (held && square) copy_transforms(A.get(), N, held, N, k, s);
    else ntt3_forward_operand(A.get(), k, a, na, s);
    if (!square && !held) ntt3_forward_operand(B.get(), k, b, nb, s);
    ntt3_pointwise(A.get(), held ? held : (square ? A.get() : B.get()), k, s);
    ntt3_inverse_to_words(A.get(), k, ncoef, 1, z, zw, s);
}

// ---- the FP64 three-prime form ---------------------------------------------
// Operands in 56-bit pieces (piece j = bits 56 j .. 56 j + 55), residues
// modulo kDblPrimes held as doubles (fp64mod.cuh), the same transform passes
// with FP64 butterflies, pointwise products without a Montgomery factor, and a
// CRT that places coefficient j (below p0 p1 p2 < 2^141) at bit 56 j.  Inverse
// outputs arrive with |y| < 12 p (unscaled).

size_t pieces56(size_t nwords) { return (32 * nwords + 55) / 56; }

struct DblPrimes3 {
    double p[3], pinv[3];
};

static DblPrimes3 dbl_primes3()
{
    DblPrimes3 d;
    for (int q = 0; q < 3; q++) {
        d.p[q] = (double)kDblPrimes[q];
        d.pinv[q] = 1.0 / d.p[q];
    }
    return d;
}

static NttBatch ntt3d_batch_stride(uint64_t* data, size_t stride)
{
    NttBatch bat;
    bat.data = data;
    bat.stride = stride;
    bat.count = 3;
    bat.per_prime = 1;
    for (int q = 0; q < 3; q++) bat.prime[q] = dbl_prime_tables(kDblPrimes[q]).dev;
    return bat;
}

// out[q stride + j] = piece first + j of a mod p_q, j < N.
__global__ void split3d_off_kernel(uint64_t* __restrict__ out, size_t stride, const uint32_t* __restrict__ a,
                                   uint32_t na, size_t first, size_t N, DblPrimes3 P)
{
    for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < N; j += (size_t)gridDim.x * blockDim.x) {
        const uint64_t v = src_piece56_raw(a, na, first + j);
#pragma unroll
        for (int q = 0; q < 3; q++) out[q * stride + j] = dstore(dpiece56(v, P.p[q], P.pinv[q]));
    }
}

static void split3d(uint64_t* out, size_t stride, const uint32_t* a, size_t na, size_t first, size_t N,
                    cudaStream_t s)
{
    PIC_REQUIRE(na < ((size_t)1 << 32), PIC_ERR_LENGTH, "operand too long for the FP64 form");
    split3d_off_kernel<<<grid_for(N, 256), 256, 0, s>>>(out, stride, a, (uint32_t)na, first, N, dbl_primes3());
    PIC_CHECK_LAUNCH();
    count_launch();
}

void ntt3d_forward_operand(uint64_t* out, int k, const uint32_t* a, size_t na, cudaStream_t s)
{
    const size_t N = (size_t)1 << k;
    {
        ProfScope ps(KC_SPLIT, 4.0 * (double)na + 24.0 * (double)N, s);
        split3d(out, N, a, na, 0, N, s);
    }
    ntt_forward_dif(ntt3d_batch_stride(out, N), k, s);
}

struct CrtDConsts {
    double p[3], pinv[3];
    double sw[3], swp[3];  // N^-1 mod p_q and its companion
    double i01, i01p;      // p0^-1 mod p1
    double i012, i012p;    // (p0 p1)^-1 mod p2
    double q012, q012p;    // p1^-1 mod p2 = p0 (p0 p1)^-1 mod p2
    double off[3];         // 2^140 mod p_q when every coefficient gets the offset 2^140, else 0
    uint64_t p0, p01_lo, p01_hi;
};

static void dbl_pair(uint64_t w, uint64_t p, double& d, double& dp)
{
    d = (double)w;
    dp = d / (double)p;
}

static CrtDConsts make_crtd(int k, bool offset)
{
    CrtDConsts C;
    const uint64_t P0 = kDblPrimes[0], P1 = kDblPrimes[1], P2 = kDblPrimes[2];
    for (int q = 0; q < 3; q++) {
        const uint64_t p = kDblPrimes[q];
        C.p[q] = (double)p;
        C.pinv[q] = 1.0 / C.p[q];
        dbl_pair(host_powmod(((uint64_t)1 << k) % p, p - 2, p), p, C.sw[q], C.swp[q]);
        C.off[q] = offset ? (double)host_powmod(2, 140, p) : 0.0;
    }
    dbl_pair(host_powmod(P0 % P1, P1 - 2, P1), P1, C.i01, C.i01p);
    dbl_pair(host_powmod(host_mulmod(P0 % P2, P1 % P2, P2), P2 - 2, P2), P2, C.i012, C.i012p);
    dbl_pair(host_powmod(P1 % P2, P2 - 2, P2), P2, C.q012, C.q012p);
    const unsigned __int128 p01 = (unsigned __int128)P0 * P1;
    C.p0 = P0;
    C.p01_lo = (uint64_t)p01;
    C.p01_hi = (uint64_t)(p01 >> 64);
    return C;
}

// x in (-p, 2p) -> [0, p)
__device__ __forceinline__ double dcanon2(double x, double p)
{
    x = x < 0.0 ? __dadd_rn(x, p) : x;
    return x >= p ? __dadd_rn(x, -p) : x;
}

// Garner's CRT on three FP64 residues (|y| < 2^51): x = r0 + p0 (v1 + p1 v2)
// with r_q = y_q N^-1 (+ offset) mod p_q, as three 64-bit limbs (x < 2^141).
__device__ __forceinline__ void crt3d(const CrtDConsts& C, double y0, double y1, double y2, uint64_t& l0,
                                      uint64_t& l1, uint64_t& l2)
{
    const double r0 = dcanon2(__dadd_rn(dmul_tw(y0, C.sw[0], C.swp[0], C.p[0]), C.off[0]), C.p[0]);
    const double r1 = dcanon2(__dadd_rn(dmul_tw(y1, C.sw[1], C.swp[1], C.p[1]), C.off[1]), C.p[1]);
    const double r2 = dcanon2(__dadd_rn(dmul_tw(y2, C.sw[2], C.swp[2], C.p[2]), C.off[2]), C.p[2]);
    const double v1 = dcanon(dmul_tw(__dadd_rn(r1, -r0), C.i01, C.i01p, C.p[1]), C.p[1]);
    const double a = dmul_tw(__dadd_rn(r2, -r0), C.i012, C.i012p, C.p[2]);
    const double b = dmul_tw(v1, C.q012, C.q012p, C.p[2]);
    const double v2 = dcanon(dreduce(__dadd_rn(a, -b), C.p[2], C.pinv[2]), C.p[2]);
    const uint64_t R0 = dto_u64(r0), V1 = dto_u64(v1), V2 = dto_u64(v2);
    const unsigned __int128 lo = (unsigned __int128)R0 + (unsigned __int128)C.p0 * V1 +
                                 (unsigned __int128)C.p01_lo * V2;  // < 2^95 + 2^111
    const unsigned __int128 hi = (lo >> 64) + (unsigned __int128)C.p01_hi * V2;
    l0 = (uint64_t)lo;
    l1 = (uint64_t)hi;
    l2 = (uint64_t)(hi >> 64);
}

// A thread takes 8 consecutive coefficients (group u: bits 448 u .. 448 u +
// 447 of the product) and the 7 limbs they start; limb L of the group
// collects the windows of the group's coefficients c = -3 .. 7 that reach it
// (coefficient c at bit 56 c, limb L at bit 64 L; c < 0 come from the
// previous thread through shared memory), so every shift is a compile-time
// constant and the lanes of a warp never diverge.
constexpr int kCrtDThreads = 128;
constexpr size_t kCrtDLPC = 7 * (size_t)kCrtDThreads;  // limbs per CTA
constexpr size_t kCrtDWPC = 2 * kCrtDLPC;

// The 64 bits of coefficient x (three limbs, below 2^141) that fall in a limb
// starting s = 56 C - 64 L bits below the coefficient's bit 0.
template <int C, int L>
__device__ __forceinline__ uint64_t coef_win(const uint64_t (&x)[3])
{
    constexpr int s = 56 * C - 64 * L;
    if constexpr (s >= 0) {
        return x[0] << s;
    } else {
        constexpr int r = -s;
        if constexpr (r < 64) return (x[0] >> r) | (x[1] << (64 - r));
        else if constexpr (r == 64) return x[1];
        else if constexpr (r < 128) return (x[1] >> (r - 64)) | (x[2] << (128 - r));
        else if constexpr (r == 128) return x[2];
        else return x[2] >> (r - 128);
    }
}

template <int L, int C = -3>
__device__ __forceinline__ void group_limb(const uint64_t (&c)[11][3], uint64_t& lo, uint64_t& hi)
{
    if constexpr (C <= 7) {
        constexpr int s = 56 * C - 64 * L;
        if constexpr (s < 64 && s > -141) add128(lo, hi, coef_win<C, L>(c[C + 3]));
        group_limb<L, C + 1>(c, lo, hi);
    }
}

template <int L>
__device__ __forceinline__ void group_limbs(const uint64_t (&c)[11][3], uint64_t (&lo)[8], uint64_t (&hi)[8])
{
    if constexpr (L <= 6) {
        lo[L + 1] = 0;
        hi[L + 1] = 0;
        group_limb<L>(c, lo[L + 1], hi[L + 1]);
        group_limbs<L + 1>(c, lo, hi);
    }
}

__device__ __forceinline__ void crt3d_block(const uint64_t* __restrict__ Y, size_t pstride, size_t ncoef,
                                            const CrtDConsts& C, uint32_t* __restrict__ z, size_t zw, int64_t cta,
                                            uint32_t* agg_slot)
{
    __shared__ uint64_t prev[kCrtDThreads][9];
    const int64_t u = cta * kCrtDThreads + threadIdx.x;
    const int64_t j0 = 8 * u;
    const int64_t climit = (int64_t)((32 * zw + 55) / 56);  // coefficients below the last word
    const int64_t jlim = climit < (int64_t)ncoef ? climit : (int64_t)ncoef;
    auto coef = [&](int64_t j, uint64_t (&x)[3]) {
        x[0] = x[1] = x[2] = 0;
        if (j >= 0 && j < jlim)
            crt3d(C, dbits(Y[j]), dbits(Y[pstride + j]), dbits(Y[2 * pstride + j]), x[0], x[1], x[2]);
    };
    uint64_t c[11][3];
#pragma unroll
    for (int i = 0; i < 8; i++) coef(j0 + i, c[3 + i]);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int w = 0; w < 3; w++) prev[threadIdx.x][3 * i + w] = c[8 + i][w];
    __syncthreads();
    if (threadIdx.x > 0) {
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int w = 0; w < 3; w++) c[i][w] = prev[threadIdx.x - 1][3 * i + w];
    } else {
#pragma unroll
        for (int i = 0; i < 3; i++) coef(j0 - 3 + i, c[i]);
    }
    uint64_t lo[8], hi[8];  // limbs -1 .. 6 of the group
    lo[0] = 0;
    hi[0] = 0;
    group_limb<-1>(c, lo[0], hi[0]);
    group_limbs<0>(c, lo, hi);
    uint64_t dig[7];
    uint32_t gen[7];
#pragma unroll
    for (int L = 0; L < 7; L++) {
        const uint64_t d = lo[L + 1] + hi[L];
        dig[L] = d;
        gen[L] = d < lo[L + 1];
    }
    const size_t zend = 2 * ((size_t)cta * kCrtDLPC + kCrtDLPC);
    limbs_to_words<7>(dig, gen, 7 * (size_t)u, z, zw < zend ? zw : zend, agg_slot);
}

__global__ void __launch_bounds__(kCrtDThreads) crt3d_k1(const uint64_t* __restrict__ Y, size_t pstride,
                                                         size_t ncoef, CrtDConsts C, uint32_t* __restrict__ z,
                                                         size_t zw, uint32_t* agg)
{
    crt3d_block(Y, pstride, ncoef, C, z, zw, (int64_t)blockIdx.x, agg + blockIdx.x);
}

__global__ void __launch_bounds__(kCrtDThreads) crt3d_batch_k1(const uint64_t* __restrict__ Y, size_t istride,
                                                               size_t pstride, size_t ncoef, CrtDConsts C,
                                                               uint32_t* __restrict__ z, uint32_t zcap,
                                                               const uint32_t* __restrict__ zlen, size_t cpp,
                                                               uint32_t* agg)
{
    const size_t prod = blockIdx.x / cpp, lc = blockIdx.x % cpp;
    crt3d_block(Y + prod * istride, pstride, ncoef, C, z + prod * (size_t)zcap, zlen[prod], (int64_t)lc,
                agg + blockIdx.x);
}

static size_t crt3d_ctas(size_t zw) { return ((zw + 1) / 2 + kCrtDLPC - 1) / kCrtDLPC; }

// Inverse-transformed residues (product length 2^k, prime q at y + q pstride)
// -> zw words.
static void crt3d_to_words(const uint64_t* y, size_t pstride, int k, size_t ncoef, uint32_t* z, size_t zw,
                           cudaStream_t s)
{
    const CrtDConsts C = make_crtd(k, false);
    const size_t nctas = crt3d_ctas(zw);
    DevBuf<uint32_t> agg(nctas, s);
    ProfScope ps(KC_CRT, 24.0 * (double)ncoef + 4.0 * (double)zw, s);
    crt3d_k1<<<(unsigned)nctas, kCrtDThreads, 0, s>>>(y, pstride, ncoef, C, z, zw, agg.get());
    PIC_CHECK_LAUNCH();
    count_launch();
    carry_scan_aggregates(agg.get(), nctas, nullptr, s);
    carry_ripple(z, zw, kCrtDWPC, agg.get(), nctas, kCarryAdd, s);
}

void ntt3d_batch_to_words(const uint64_t* y, size_t istride, size_t pstride, size_t count, int k, uint32_t* z,
                          uint32_t zcap, const uint32_t* zlen, cudaStream_t s, size_t ncoef, bool offset)
{
    if (count == 0) return;
    if (ncoef == 0) ncoef = (size_t)1 << k;
    const CrtDConsts C = make_crtd(k, offset);
    const size_t cpp = crt3d_ctas(zcap);
    const size_t nctas = count * cpp;
    DevBuf<uint32_t> agg(nctas, s);
    {
        ProfScope ps(KC_CRT, (24.0 * (double)ncoef + 4.0 * zcap) * (double)count, s);
        crt3d_batch_k1<<<(unsigned)nctas, kCrtDThreads, 0, s>>>(y, istride, pstride, ncoef, C, z, zcap, zlen, cpp,
                                                               agg.get());
        PIC_CHECK_LAUNCH();
        count_launch();
    }
    carry_scan_segments(agg.get(), count, cpp, s);
    carry_ripple_batch(z, zcap, zlen, kCrtDWPC, agg.get(), count, cpp, s);
}

// The wrapped form's fix-up (see wrap_fix_kernel) on FP64 residues:
// y[j] -= h, y[Nm + j] = h with h = d_(W-1+j) Nm / T mod p.
__global__ void wrap_fix_d_kernel(uint64_t* __restrict__ y, size_t ystride, const uint64_t* __restrict__ tail,
                                  size_t T, size_t nitems, size_t item_mul, size_t nchild, size_t Nm, size_t W,
                                  DblPrimes3 P, double cw, double cwp0, double cwp1, double cwp2)
{
    const size_t total = 3 * nitems * W;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < total; g += (size_t)gridDim.x * blockDim.x) {
        const size_t q = g / (nitems * W);
        const size_t r = g - q * nitems * W;
        const size_t it = r / W, j = r - it * W;
        const double p = q == 0 ? P.p[0] : (q == 1 ? P.p[1] : P.p[2]);
        const double wp = q == 0 ? cwp0 : (q == 1 ? cwp1 : cwp2);
        const size_t child = q * nchild + it * item_mul;
        const double h = dmul_tw(dbits(tail[child * T + W - 1 + j]), cw, wp, p);
        uint64_t* yi = y + child * ystride;
        yi[j] = dstore(__dadd_rn(dbits(yi[j]), -h));
        yi[Nm + j] = dstore(h);
    }
}

void launch_wrap_fix_d(uint64_t* y, size_t ystride, const uint64_t* tail, size_t T, size_t nitems,
                       size_t item_mul, size_t nchild, size_t Nm, size_t W, cudaStream_t s)
{
    const double cw = (double)(Nm / T);  // below every prime
    wrap_fix_d_kernel<<<grid_for(3 * nitems * W, 256), 256, 0, s>>>(
        y, ystride, tail, T, nitems, item_mul, nchild, Nm, W, dbl_primes3(), cw, cw / (double)kDblPrimes[0],
        cw / (double)kDblPrimes[1], cw / (double)kDblPrimes[2]);
    PIC_CHECK_LAUNCH();
}

// Largest shorter operand (in pieces) the FP64 form multiplies exactly:
// coefficients below 2^28 (2^56 - 1)^2 < p0 p1 p2.
constexpr size_t kDblMaxPieces = (size_t)1 << 28;

static void mul_ntt3d_wrapped(uint32_t* z, const uint32_t* a, size_t na, const uint32_t* b, size_t nb, int km,
                              int kt, cudaStream_t s)
{
    const size_t zw = na + nb;
    const size_t pa = pieces56(na), pb = pieces56(nb);
    const size_t L = pa + pb - 1;
    const size_t Nm = (size_t)1 << km, T = (size_t)1 << kt, W = L - Nm;
    const size_t ST = Nm + ((W + 15) & ~(size_t)15);
    const bool square = (a == b && na == nb);
    const uint64_t* held = is_held(b, nb) ? held_transform(km, kFormDbl, s) : nullptr;
    DevBuf<uint64_t> A(3 * ST, s), B(square || held ? 0 : 3 * ST, s), tA(3 * T, s), tB(square ? 0 : 3 * T, s);
    {
        ProfScope ps(KC_SPLIT, 4.0 * (double)(na + nb) + 24.0 * (double)(2 * (Nm + T)), s);
        if (!(held && square)) split3d(A.get(), ST, a, na, 0, Nm, s);
        split3d(tA.get(), T, a, na, Nm - pb + 1, T, s);
        if (!square) {
            if (!held) split3d(B.get(), ST, b, nb, 0, Nm, s);
            split3d(tB.get(), T, b, nb, Nm - pa + 1, T, s);
        }
    }
    const NttBatch mA = ntt3d_batch_stride(A.get(), ST), mB = ntt3d_batch_stride(B.get(), ST);
    const NttBatch xA = ntt3d_batch_stride(tA.get(), T), xB = ntt3d_batch_stride(tB.get(), T);
    if (held && square) copy_transforms(A.get(), ST, held, Nm, km, s);
    else ntt_forward_dif(mA, km, s);
    ntt_forward_dif(xA, kt, s);
    if (!square) {
        if (!held) ntt_forward_dif(mB, km, s);
        ntt_forward_dif(xB, kt, s);
    }
    if (held) ntt_pointwise_mont(mA, held, km, s, Nm);
    else ntt_pointwise_mont(mA, square ? A.get() : B.get(), km, s);
    ntt_pointwise_mont(xA, square ? tA.get() : tB.get(), kt, s);
    ntt_inverse_dit(mA, km, s);
    ntt_inverse_dit(xA, kt, s);
    {
        ProfScope ps(KC_NTT_POINTWISE, 3.0 * (double)W * 24.0, s);
        launch_wrap_fix_d(A.get(), ST, tA.get(), T, 1, 1, 1, Nm, W, s);
        count_launch();
    }
    crt3d_to_words(A.get(), ST, km, L, z, zw, s);
}

// The FP64 form of mul_ntt3 (PIC_MUL_NTT3D): products whose shorter operand
// has more than 2^28 pieces go to the integer form.
void mul_ntt3d(uint32_t* z, const uint32_t* a, size_t na, const uint32_t* b, size_t nb, cudaStream_t s)
{
    if (is_held(a, na) && !(a == b && na == nb)) {  // the held operand goes second
        std::swap(a, b);
        std::swap(na, nb);
    }
    const size_t zw = na + nb;
    const size_t pa = pieces56(na), pb = pieces56(nb);
    if ((pa < pb ? pa : pb) > kDblMaxPieces) {
        mul_ntt3(z, a, na, b, nb, s);
        return;
    }
    const size_t ncoef = pa + pb - 1;
    int k = ceil_log2(ncoef);
    if (k < 1) k = 1;
    PIC_REQUIRE(k <= 30, PIC_ERR_LENGTH, "product too long for the FP64 three-prime NTT (2^30 points)");
    const size_t N = (size_t)1 << k;
    if (g_mul_wrap && k >= 4) {
        const size_t Nm = N / 2;
        if (std::max(pa, pb) <= Nm && ncoef > Nm) {
            const size_t W = ncoef - Nm;
            int kt = ceil_log2(2 * W - 1);
            if (kt < 2) kt = 2;
            if (((size_t)1 << kt) <= Nm / 2) {
                mul_ntt3d_wrapped(z, a, na, b, nb, k - 1, kt, s);
                return;
            }
        }
    }
    const bool square = (a == b && na == nb);
    const uint64_t* held = is_held(b, nb) ? held_transform(k, kFormDbl, s) : nullptr;
    DevBuf<uint64_t> A(3 * N, s);
    DevBuf<uint64_t> B(square || held ? 0 : 3 * N, s);
    if (held && square) copy_transforms(A.get(), N, held, N, k, s);
    else ntt3d_forward_operand(A.get(), k, a, na, s);
    if (!square && !held) ntt3d_forward_operand(B.get(), k, b, nb, s);
    ntt_pointwise_mont(ntt3d_batch_stride(A.get(), N), held ? held : (square ? A.get() : B.get()), k, s);
    ntt_inverse_dit(ntt3d_batch_stride(A.get(), N), k, s);
    crt3d_to_words(A.get(), N, k, ncoef, z, zw, s);
}

void mul_ntt_ref(uint32_t* z, const uint32_t* a, size_t na, const uint32_t* b, size_t nb, cudaStream_t s)
{
    const size_t zw = na + nb;
    int k = ceil_log2(4 * zw);  // BigFloat.cpp:380-385
    PIC_REQUIRE(k <= 32, PIC_ERR_LENGTH, "product too long for the reference layout");
    const size_t N = (size_t)1 << k;
    const uint64_t p = reference_prime(k);
    const PrimeDev P = prime_tables(p).dev;
    const bool square = (a == b && na == nb);
    NttBatch bat;
    bat.stride = N;
    bat.count = 1;
    bat.per_prime = 1;
    bat.prime[0] = P;
    DevBuf<uint64_t> A(N, s), B(square ? 0 : N, s);
    split16_kernel<<<grid_for(N, 256), 256, 0, s>>>(A.get(), N, a, na);
    PIC_CHECK_LAUNCH();
    count_launch();
    bat.data = A.get();
    ntt_forward_dif(bat, k, s);
    if (!square) {
        split16_kernel<<<grid_for(N, 256), 256, 0, s>>>(B.get(), N, b, nb);
        PIC_CHECK_LAUNCH();
        count_launch();
        NttBatch bb = bat;
        bb.data = B.get();
        ntt_forward_dif(bb, k, s);
    }
    ntt_pointwise_mont(bat, square ? A.get() : B.get(), k, s);
    ntt_inverse_dit(bat, k, s);
    const uint64_t ninv = host_powmod(N % p, p - 2, p);
    coef16_to_words(A.get(), 2 * zw, to_mont(to_mont(ninv, p), p), p, P.pinv_neg, z, zw, s);
}

// ---- schoolbook ----------------------------------------------------------------
// One CTA per product.  Phase 1: column sums v_c = sum a_i b_(c-i) as 96-bit
// (3 words) in shared memory, columns dealt round-robin.  Phase 2: each thread
// owns kSchWPT consecutive output words: S_w = v_w.0 + v_(w-1).1 + v_(w-2).2.
constexpr int kSchThreads = 256;
constexpr int kSchWPT = (int)(kSchoolMaxWords / kSchThreads);

__global__ void __launch_bounds__(kSchThreads) school_kernel(uint32_t* __restrict__ z, const uint32_t* __restrict__ a,
                                                             uint32_t na, const uint32_t* __restrict__ b, uint32_t nb)
{
    extern __shared__ uint32_t sm[];
    uint32_t* sa = sm;
    uint32_t* sb = sa + na;
    uint32_t* col = sb + nb;  // 3 words per column, columns 0 .. na+nb-1
    const uint32_t zw = na + nb;
    for (uint32_t i = threadIdx.x; i < na; i += blockDim.x) sa[i] = a[i];
    for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) sb[i] = b[i];
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < zw; c += blockDim.x) {
        uint64_t lo = 0;
        uint32_t hi = 0;
        const uint32_t i_lo = c + 1 > nb ? c + 1 - nb : 0;
        const uint32_t i_hi = c < na - 1 ? c : na - 1;
        for (uint32_t i = i_lo; i <= i_hi && c + 1 < zw + 1; i++) {
            const uint64_t pr = (uint64_t)sa[i] * sb[c - i];
            lo += pr;
            hi += (lo < pr);
        }
        if (i_lo > i_hi) { lo = 0; hi = 0; }
        col[3 * c] = (uint32_t)lo;
        col[3 * c + 1] = (uint32_t)(lo >> 32);
        col[3 * c + 2] = hi;
    }
    __syncthreads();
    uint32_t d[kSchWPT], gg[kSchWPT];
    uint32_t gp = kGPIdentity;
    const uint32_t w0 = threadIdx.x * kSchWPT;
#pragma unroll 4
    for (int u = 0; u < kSchWPT; u++) {
        const uint32_t w = w0 + u;
        uint32_t dig = 0, g = 0;
        if (w < zw) {
            uint64_t sw = col[3 * w];
            uint64_t sp = 0;
            if (w >= 1) { sw += col[3 * (w - 1) + 1]; sp += col[3 * (w - 1)]; }
            if (w >= 2) { sw += col[3 * (w - 2) + 2]; sp += col[3 * (w - 2) + 1]; }
            if (w >= 3) sp += col[3 * (w - 3) + 2];
            const uint64_t t = (sw & 0xffffffffu) + (sp >> 32);
            dig = (uint32_t)t;
            g = (uint32_t)(t >> 32);
        }
        d[u] = dig;
        gg[u] = g;
        if (w < zw) gp = gp_combine(gp, g | ((uint32_t)(dig == 0xffffffffu) << 1));
    }
    uint32_t total;
    uint32_t cin = block_gp_scan(gp, &total) & 1u;
#pragma unroll 4
    for (int u = 0; u < kSchWPT; u++) {
        const uint32_t w = w0 + u;
        if (w < zw) z[w] = d[u] + cin;
        cin = gg[u] | ((uint32_t)(d[u] == 0xffffffffu) & cin);
    }
}

void mul_school(uint32_t* z, const uint32_t* a, size_t na, const uint32_t* b, size_t nb, cudaStream_t s)
{
    PIC_REQUIRE(na + nb <= kSchoolMaxWords, PIC_ERR_INVALID, "schoolbook product too long");
    const size_t smem = (na + nb) * 4 + (na + nb) * 12;
    if (smem > 48 * 1024)
        PIC_CUDA(cudaFuncSetAttribute(school_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    ProfScope ps(KC_SCHOOL, 4.0 * (double)(2 * (na + nb)), s);
    school_kernel<<<1, kSchThreads, smem, s>>>(z, a, (uint32_t)na, b, (uint32_t)nb);
    PIC_CHECK_LAUNCH();
    count_launch();
}

// ---- dispatch ------------------------------------------------------------------
static int64_t g_school_max_words = 256;
static int64_t g_fft_max_words = 0;

void mul_set_thresholds(int64_t school_max, int64_t fft_max)
{
    if (school_max >= 0) g_school_max_words = school_max;
    if (fft_max >= 0) g_fft_max_words = fft_max;
}
int64_t mul_school_max() { return g_school_max_words; }
int64_t mul_fft_max() { return g_fft_max_words; }

// The three-prime form AUTO and the binary splitting use: kFormInt,
// kFormDbl, or kFormChosen (per product, the form with less transform work).
static int g_ntt_form = kFormInt;
void mul_set_ntt_form(int form)
{
    PIC_REQUIRE(form == kFormInt || form == kFormDbl || form == kFormChosen, PIC_ERR_INVALID,
                "unknown product form");
    g_ntt_form = form;
}
int mul_ntt_form() { return g_ntt_form; }

// Butterfly work (sum of N log2 N over the transforms) of a three-prime
// product with `coefs` coefficients and operands of at most per_max pieces,
// under the plain / wrapped rule of mul_ntt3 and mul_ntt3d.
static double ntt_work(size_t coefs, size_t per_max, bool wrap)
{
    int k = ceil_log2(coefs);
    if (k < 1) k = 1;
    const size_t N = (size_t)1 << k;
    if (wrap && k >= 4) {
        const size_t Nm = N / 2;
        if (per_max <= Nm && coefs > Nm) {
            int kt = ceil_log2(2 * (coefs - Nm) - 1);
            if (kt < 2) kt = 2;
            if (((size_t)1 << kt) <= Nm / 2) return (double)Nm * (k - 1) + (double)((size_t)1 << kt) * kt;
        }
    }
    return (double)N * k;
}

// The FP64 form's cost per butterfly relative to the integer form's, at equal
// transform length (isolated products of 2^20 .. 2^26 points: 0.83 - 0.90).
constexpr double kDblWorkRatio = 0.87;

int ntt_form_for(size_t pieces_int_a, size_t pieces_int_b, size_t pieces_dbl_a, size_t pieces_dbl_b, bool wrap)
{
    if (g_ntt_form != kFormChosen) return g_ntt_form;
    const double wi = ntt_work(pieces_int_a + pieces_int_b - 1, std::max(pieces_int_a, pieces_int_b), wrap);
    const double wd = ntt_work(pieces_dbl_a + pieces_dbl_b - 1, std::max(pieces_dbl_a, pieces_dbl_b), wrap);
    return wd * kDblWorkRatio < wi ? kFormDbl : kFormInt;
}

static int product_form(size_t na, size_t nb)
{
    return ntt_form_for((na + 1) / 2, (nb + 1) / 2, pieces56(na), pieces56(nb), g_mul_wrap);
}

int mul_auto_mode(size_t na, size_t nb)
{
    const size_t mn = na < nb ? na : nb;
    const size_t zw = na + nb;
    if (zw <= kSchoolMaxWords && (mn <= 48 || (int64_t)zw <= g_school_max_words)) return PIC_MUL_SCHOOL;
    if ((int64_t)zw <= g_fft_max_words) return PIC_MUL_FFT;
    return product_form(na, nb) == kFormDbl ? PIC_MUL_NTT3D : PIC_MUL_NTT3;
}

static std::atomic<uint64_t> g_fft_err_bits{0};
static std::atomic<uint64_t> g_fft_err_max_bits{0};  // largest since fft_reset_max_err
double fft_last_max_err()
{
    uint64_t b = g_fft_err_bits.load();
    double d;
    memcpy(&d, &b, sizeof d);
    return d;
}
double fft_max_err_seen()
{
    uint64_t b = g_fft_err_max_bits.load();
    double d;
    memcpy(&d, &b, sizeof d);
    return d;
}
void fft_reset_max_err() { g_fft_err_max_bits.store(0); }
void fft_note_max_err(double e)
{
    uint64_t b;
    memcpy(&b, &e, sizeof b);
    g_fft_err_bits.store(b);
    // nonnegative doubles order like their bit patterns
    uint64_t cur = g_fft_err_max_bits.load();
    while (b > cur && !g_fft_err_max_bits.compare_exchange_weak(cur, b)) {
    }
}

// Largest accepted distance to the nearest integer of an FFT product's
// coefficients; past it the product is recomputed with the three-prime NTT.
// 0.25 is the production value; tests lower it to force the recompute.
static double g_fft_accept = 0.25;
void mul_set_fft_accept(double max_dist) { g_fft_accept = max_dist; }
double mul_fft_accept() { return g_fft_accept; }

void mul_dispatch(uint32_t* z, const uint32_t* a, size_t na, const uint32_t* b, size_t nb, int mode,
                  cudaStream_t s)
{
    PIC_REQUIRE(na > 0 && nb > 0, PIC_ERR_INVALID, "empty operand");
    if (mode == PIC_MUL_AUTO) mode = mul_auto_mode(na, nb);
    count_products(1);
    switch (mode) {
    case PIC_MUL_SCHOOL:
        if (na + nb <= kSchoolMaxWords) {
            mul_school(z, a, na, b, nb, s);
            return;
        }
        mul_ntt3(z, a, na, b, nb, s);
        return;
    case PIC_MUL_NTT_REF: mul_ntt_ref(z, a, na, b, nb, s); return;
    case PIC_MUL_NTT3: mul_ntt3(z, a, na, b, nb, s); return;
    case PIC_MUL_NTT3D: mul_ntt3d(z, a, na, b, nb, s); return;
    case PIC_MUL_FFT: {
        double e = 0;
        if (!mul_fft(z, a, na, b, nb, s, &e) || e > g_fft_accept) {
            // the NTT is the oracle: a product whose rounding distance passed
            // the acceptance threshold is redone exactly
            ctx().fft_recomputes.fetch_add(1);
            if (product_form(na, nb) == kFormDbl) mul_ntt3d(z, a, na, b, nb, s);
            else mul_ntt3(z, a, na, b, nb, s);
        }
        return;
    }
    default: throw Error(PIC_ERR_INVALID, "unknown multiply mode");
    }
}

// ---- reference-API conversions ---------------------------------------------------
void int_to_ntt_dev(uint64_t* T, int k, const uint32_t* A, size_t AL, cudaStream_t s)
{
    const size_t N = (size_t)1 << k;
    PIC_REQUIRE(2 * AL <= N, PIC_ERR_LENGTH, "FFT length is too small.");
    split16_kernel<<<grid_for(N, 256), 256, 0, s>>>(T, N, A, AL);
    PIC_CHECK_LAUNCH();
    count_launch();
}

void ntt_to_int_dev(const uint64_t* T, int k, uint32_t* A, size_t AL, cudaStream_t s)
{
    const size_t N = (size_t)1 << k;
    PIC_REQUIRE(N >= 2 * AL, PIC_ERR_LENGTH, "FFT length is too small.");  // NTT.cpp:352-353
    coef16_to_words(T, 2 * AL, 0, 0, 0, A, AL, s);
}

}  // namespace pic
