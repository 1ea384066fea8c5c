// pic_mul_noalloc: an exact three-prime NTT product that allocates nothing.
//
// Who needs it: callers that cannot call cudaMalloc at the moment they
// multiply -- for instance an application that has already handed almost all
// device memory to its own pool allocator, or a latency-critical loop that
// must not take the CUDA allocator's locks nor risk an out-of-memory failure
// halfway through a computation.  pic_mul takes its transform buffers from the
// stream-ordered pool; this entry point instead uses fixed storage compiled
// into the library:
//   * g_residues: the two operands' residues, 2 x 3 x 2^16 uint64 (3 MiB);
//   * g_carry:    the per-CTA carry aggregates of the word conversion;
//   * g_tables:   twiddle tables for the three primes, roots of order 2^16.
// Every GPU that loads the library holds these arrays (about 3.5 MiB) until
// the process exits.  The product length limit is therefore
//   ceil(na / 2) + ceil(nb / 2) - 1 <= 65536 points (about 131,000 words of
//   product); longer products are rejected with PIC_ERR_LENGTH.
// All calls share the arrays: two calls that overlap on the GPU (different
// streams, or different host threads on one device) race and corrupt each
// other's results.  Every buffer is fully written before it is read within
// a call (the split writes all 2^k residues including the zero padding), so
// no clearing is needed between calls.  The tables hold only the two-level
// roots, not the per-level and per-pass tables of pic_mul (pass tables are
// allocated on first use), so these transforms run on the general NTT
// kernels: the same words as pic_mul, somewhat slower.
#include <stdio.h>

#include <mutex>

#include "common.cuh"
#include "mul.cuh"
#include "ntt.cuh"

namespace pic {

constexpr int kNoallocK = 16;                                  // largest transform, 2^16 points
constexpr size_t kNoallocN = (size_t)1 << kNoallocK;
constexpr int kNoallocS = kNoallocK / 2;                       // outer table split
constexpr size_t kInnerPairs = (size_t)1 << (kInnerBits - 1);  // Shoup pairs per inner table
// per prime: inner fwd + inner inv (pairs), outer lo/hi fwd/inv
constexpr size_t kTablePerPrime = 2 * 2 * kInnerPairs + 4 * ((size_t)1 << kNoallocS);
constexpr size_t kNoallocCarry = kNoallocN / 256 + 8;  // >= crt3_scratch_ctas(2 * kNoallocN + 2)

static __device__ __align__(256) uint64_t g_residues[2 * 3 * kNoallocN];
static __device__ __align__(256) uint32_t g_carry[kNoallocCarry];
static __device__ __align__(256) uint64_t g_tables[3 * kTablePerPrime];

// Fills one prime's tables: w = g^((p-1)/2^16) (a primitive 2^16-th root).
__global__ void noalloc_tables_kernel(uint64_t* tab, uint64_t p, uint64_t pinv, uint64_t r2, uint64_t w_mont,
                                      uint64_t wi_mont)
{
    const uint64_t one_m = mont_mul(1, r2, p, pinv);  // R mod p
    auto mpow = [&](uint64_t base_m, uint64_t e) {
        uint64_t r = one_m, b = base_m;
        while (e) {
            if (e & 1) r = mont_mul(r, b, p, pinv);
            b = mont_mul(b, b, p, pinv);
            e >>= 1;
        }
        return r;  // Montgomery form
    };
    const size_t nlo = (size_t)1 << kNoallocS;
    uint64_t* in_f = tab;
    uint64_t* in_i = in_f + 2 * kInnerPairs;
    uint64_t* lo_f = in_i + 2 * kInnerPairs;
    uint64_t* hi_f = lo_f + nlo;
    uint64_t* lo_i = hi_f + nlo;
    uint64_t* hi_i = lo_i + nlo;
    const uint64_t step = (uint64_t)1 << (kNoallocK - kInnerBits);  // inner root = w^(2^(16-13))
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < kInnerPairs; i += (size_t)gridDim.x * blockDim.x) {
        const uint64_t f = mont_mul(mpow(w_mont, i * step), 1, p, pinv);  // plain value
        const uint64_t v = mont_mul(mpow(wi_mont, i * step), 1, p, pinv);
        in_f[2 * i] = f;
        in_f[2 * i + 1] = (uint64_t)((((unsigned __int128)f) << 64) / p);
        in_i[2 * i] = v;
        in_i[2 * i + 1] = (uint64_t)((((unsigned __int128)v) << 64) / p);
    }
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nlo; i += (size_t)gridDim.x * blockDim.x) {
        lo_f[i] = mpow(w_mont, i);
        hi_f[i] = mpow(w_mont, i << kNoallocS);
        lo_i[i] = mpow(wi_mont, i);
        hi_i[i] = mpow(wi_mont, i << kNoallocS);
    }
}

namespace {
struct NoallocDevice {
    bool ready = false;
    uint64_t* residues = nullptr;
    uint32_t* carry = nullptr;
    PrimeDev prime[3];
};
std::mutex g_noalloc_lock;
NoallocDevice g_noalloc[64];
}  // namespace

// Once per device, with that device current: resolve the arrays' device
// addresses (host code may not use the symbols' host-side stand-ins) and fill
// the twiddle tables.  Runs inside the first pic_mul_noalloc call on each
// device; it synchronises that stream, so the first call belongs outside any
// stream capture.  The addresses and tables belong to the calling thread's
// current device, so that device, the stream's device and the library's
// device must all be the same one (else PIC_ERR_INVALID).
static const NoallocDevice& noalloc_setup(cudaStream_t s)
{
    int dev = 0, sdev = 0;
    PIC_CUDA(cudaGetDevice(&dev));
    PIC_CUDA(cudaStreamGetDevice(s, &sdev));
    PIC_REQUIRE(dev == ctx().device && sdev == ctx().device, PIC_ERR_INVALID,
                "pic_mul_noalloc: the current device and the stream's device must be the one given to pic_init");
    PIC_REQUIRE(dev >= 0 && dev < 64, PIC_ERR_INVALID, "device index out of range");
    std::lock_guard<std::mutex> g(g_noalloc_lock);
    NoallocDevice& d = g_noalloc[dev];
    if (d.ready) return d;
    void* res = nullptr;
    void* car = nullptr;
    void* tab = nullptr;
    PIC_CUDA(cudaGetSymbolAddress(&res, g_residues));
    PIC_CUDA(cudaGetSymbolAddress(&car, g_carry));
    PIC_CUDA(cudaGetSymbolAddress(&tab, g_tables));
    d.residues = (uint64_t*)res;
    d.carry = (uint32_t*)car;
    for (int q = 0; q < 3; q++) {
        const uint64_t p = kProductPrimes[q];
        const Mod64 m = make_mod(p);
        const uint64_t gen = smallest_generator(p);
        const uint64_t w = host_powmod(gen, (p - 1) >> kNoallocK, p);
        const uint64_t wi = host_powmod(w, p - 2, p);
        uint64_t* t = (uint64_t*)tab + q * kTablePerPrime;
        noalloc_tables_kernel<<<64, 256, 0, s>>>(t, p, m.pinv_neg, m.r2, to_mont(w, p), to_mont(wi, p));
        PIC_CHECK_LAUNCH();
        const size_t nlo = (size_t)1 << kNoallocS;
        PrimeDev& P = d.prime[q];
        P.p = p;
        P.pinv_neg = m.pinv_neg;
        P.r2 = m.r2;
        P.K = kNoallocK;
        P.S = kNoallocS;
        P.IB = kInnerBits;
        P.lazy = 1;  // the three product primes are below 2^62
        P.inner_fwd = t;
        P.inner_inv = t + 2 * kInnerPairs;
        P.olo_fwd = t + 4 * kInnerPairs;
        P.ohi_fwd = P.olo_fwd + nlo;
        P.olo_inv = P.ohi_fwd + nlo;
        P.ohi_inv = P.olo_inv + nlo;
    }
    PIC_CUDA(cudaStreamSynchronize(s));
    d.ready = true;
    return d;
}

void mul_noalloc(uint32_t* z, const uint32_t* a, size_t na, const uint32_t* b, size_t nb, cudaStream_t s)
{
    const size_t zw = na + nb;
    const size_t ncoef = (na + 1) / 2 + (nb + 1) / 2 - 1;
    PIC_REQUIRE(ncoef <= kNoallocN, PIC_ERR_LENGTH,
                "pic_mul_noalloc: product longer than the fixed scratch (65536 points)");
    int k = 1;
    while (((size_t)1 << k) < ncoef) k++;
    const NoallocDevice& d = noalloc_setup(s);
    const size_t N = (size_t)1 << k;
    PIC_REQUIRE(crt3_scratch_ctas(zw) <= kNoallocCarry, PIC_ERR_LENGTH, "pic_mul_noalloc: carry scratch too small");
    uint64_t* A = d.residues;
    uint64_t* B = d.residues + 3 * kNoallocN;
    NttBatch bat;
    bat.stride = N;
    bat.count = 3;
    bat.per_prime = 1;
    for (int q = 0; q < 3; q++) bat.prime[q] = d.prime[q];
    const bool square = (a == b && na == nb);
    split3_into(A, k, a, na, kProductPrimes, s);
    bat.data = A;
    ntt_forward_dif(bat, k, s);
    if (!square) {
        split3_into(B, k, b, nb, kProductPrimes, s);
        NttBatch bb = bat;
        bb.data = B;
        ntt_forward_dif(bb, k, s);
    }
    ntt_pointwise_mont(bat, square ? A : B, k, s);
    ntt_inverse_dit(bat, k, s);
    crt3_to_words_scratch(A, k, ncoef, z, zw, d.carry, s);
}

}  // namespace pic
