// Cross-CTA carry phases and the BigFloat linear kernels (windowed add/sub,
// multiply by a 32-bit word, leading-zero search, magnitude compare).
#include "carry.cuh"
#include "common.cuh"
#include "linear.cuh"

namespace pic {

// ---- K2: scan of per-CTA (G, P) pairs, one CTA -----------------------------
__global__ void __launch_bounds__(1024) carry_scan_kernel(uint32_t* agg, size_t n, uint32_t* final_carry)
{
    const size_t per = (n + blockDim.x - 1) / blockDim.x;
    const size_t b = threadIdx.x * per, e = b + per < n ? b + per : n;
    uint32_t acc = kGPIdentity;
    for (size_t i = b; i < e; i++) acc = gp_combine(acc, agg[i]);
    uint32_t total;
    const uint32_t pre = block_gp_scan(acc, &total);
    uint32_t cin = pre & 1u;  // carry into this segment (array carry-in 0)
    for (size_t i = b; i < e; i++) {
        const uint32_t gp = agg[i];
        agg[i] = cin;
        cin = (gp & 1u) | ((gp >> 1) & cin);
    }
    if (threadIdx.x == 0 && final_carry) *final_carry = total & 1u;
}

void carry_scan_aggregates(uint32_t* agg, size_t nctas, uint32_t* final_carry, cudaStream_t s)
{
    ProfScope ps(KC_CARRY, 8.0 * (double)nctas, s);
    carry_scan_kernel<<<1, 1024, 0, s>>>(agg, nctas, final_carry);
    PIC_CHECK_LAUNCH();
    count_launch();
}

__global__ void __launch_bounds__(256) carry_scan_seg_kernel(uint32_t* agg, size_t cpp)
{
    uint32_t* a = agg + blockIdx.x * cpp;
    const size_t per = (cpp + blockDim.x - 1) / blockDim.x;
    const size_t b = threadIdx.x * per, e = b + per < cpp ? b + per : cpp;
    uint32_t acc = kGPIdentity;
    for (size_t i = b; i < e; i++) acc = gp_combine(acc, a[i]);
    uint32_t total;
    const uint32_t pre = block_gp_scan(acc, &total);
    uint32_t cin = pre & 1u;
    for (size_t i = b; i < e; i++) {
        const uint32_t gp = a[i];
        a[i] = cin;
        cin = (gp & 1u) | ((gp >> 1) & cin);
    }
}

void carry_scan_segments(uint32_t* agg, size_t count, size_t cpp, cudaStream_t s)
{
    ProfScope ps(KC_CARRY, 8.0 * (double)(count * cpp), s);
    carry_scan_seg_kernel<<<(unsigned)count, 256, 0, s>>>(agg, cpp);
    PIC_CHECK_LAUNCH();
    count_launch();
}

__global__ void carry_ripple_batch_kernel(uint32_t* z, uint32_t zcap, const uint32_t* zlen, size_t wpc,
                                          const uint32_t* cin, size_t cpp)
{
    if (cin[blockIdx.x] == 0) return;
    const size_t prod = blockIdx.x / cpp, lc = blockIdx.x % cpp;
    uint32_t* zz = z + prod * (size_t)zcap;
    const size_t n = zlen[prod];
    const size_t b = lc * wpc, e = b + wpc < n ? b + wpc : n;
    unsigned long long mine = ~0ull;
    for (size_t i = b + threadIdx.x; i < e; i += blockDim.x)
        if (zz[i] != 0xffffffffu && i < mine) mine = i;
    const size_t f = (size_t)block_min_u64(mine);
    for (size_t i = b + threadIdx.x; i < e && i < f; i += blockDim.x) zz[i] = 0;
    if (threadIdx.x == 0 && f < e) zz[f] += 1u;
}

void carry_ripple_batch(uint32_t* z, uint32_t zcap, const uint32_t* zlen, size_t words_per_cta,
                        const uint32_t* agg_cin, size_t count, size_t cpp, cudaStream_t s)
{
    ProfScope ps(KC_CARRY, 4.0 * (double)(count * cpp), s);
    carry_ripple_batch_kernel<<<(unsigned)(count * cpp), 256, 0, s>>>(z, zcap, zlen, words_per_cta, agg_cin, cpp);
    PIC_CHECK_LAUNCH();
    count_launch();
}

// ---- K3: ripple a carry-in of 1 through one CTA's words --------------------
__global__ void carry_ripple_kernel(uint32_t* z, size_t n, size_t wpc, const uint32_t* cin, int mode)
{
    const size_t c = blockIdx.x;
    if (cin[c] == 0) return;
    const size_t b = c * wpc, e = b + wpc < n ? b + wpc : n;
    const uint32_t stop_unless = mode == kCarryAdd ? 0xffffffffu : 0u;
    unsigned long long mine = ~0ull;
    for (size_t i = b + threadIdx.x; i < e; i += blockDim.x)
        if (z[i] != stop_unless && i < mine) mine = i;
    const size_t f = (size_t)block_min_u64(mine);
    for (size_t i = b + threadIdx.x; i < e && i < f; i += blockDim.x) z[i] = ~stop_unless;
    if (threadIdx.x == 0 && f < e) z[f] = mode == kCarryAdd ? z[f] + 1u : z[f] - 1u;
}

void carry_ripple(uint32_t* z, size_t nwords, size_t words_per_cta, const uint32_t* agg_cin,
                  size_t nctas, CarryMode mode, cudaStream_t s)
{
    ProfScope ps(KC_CARRY, 4.0 * (double)nctas, s);
    carry_ripple_kernel<<<(unsigned)nctas, 256, 0, s>>>(z, nwords, words_per_cta, agg_cin, (int)mode);
    PIC_CHECK_LAUNCH();
    count_launch();
}

// ---- K1 for the linear ops --------------------------------------------------
// Each thread owns kLinIPT consecutive words; a CTA owns blockDim * kLinIPT.
constexpr int kLinIPT = 8;
constexpr int kLinThreads = 256;
constexpr size_t kLinWPC = (size_t)kLinIPT * kLinThreads;

__device__ __forceinline__ uint32_t word_at(const uint32_t* T, int64_t exp, int64_t L, int64_t mag)
{
    // BigFloat::word_at, BigFloat.cpp:109-122
    const int64_t i = mag - exp;
    return (i >= 0 && i < L) ? T[i] : 0u;
}

// Windowed add / subtract of two magnitudes: z[c] = a(bot+c) +/- b(bot+c).
__global__ void __launch_bounds__(kLinThreads) addsub_k1(uint32_t* z, size_t TL, WordView a, WordView b,
                                                         int64_t bot, int mode, uint32_t* agg)
{
    const size_t i0 = (size_t)blockIdx.x * kLinWPC + (size_t)threadIdx.x * kLinIPT;
    uint32_t d[kLinIPT], gg[kLinIPT];
    uint32_t gp = kGPIdentity;
#pragma unroll
    for (int u = 0; u < kLinIPT; u++) {
        const size_t i = i0 + u;
        uint32_t g = 0, dig = 0;
        if (i < TL) {
            const int64_t mag = bot + (int64_t)i;
            const uint32_t x = word_at(a.T, a.exp, a.L, mag), y = word_at(b.T, b.exp, b.L, mag);
            if (mode == kCarryAdd) {
                const uint64_t s = (uint64_t)x + y;
                dig = (uint32_t)s;
                g = (uint32_t)(s >> 32);
            } else {
                dig = x - y;
                g = x < y;
            }
        }
        const uint32_t p = mode == kCarryAdd ? (dig == 0xffffffffu) : (dig == 0u);
        d[u] = dig;
        gg[u] = g;
        if (i < TL) gp = gp_combine(gp, g | (p << 1));  // padding is the scan identity
    }
    uint32_t total;
    uint32_t cin = block_gp_scan(gp, &total) & 1u;
#pragma unroll
    for (int u = 0; u < kLinIPT; u++) {
        const size_t i = i0 + u;
        if (i >= TL) break;
        const uint32_t dig = d[u];
        uint32_t p;
        if (mode == kCarryAdd) {
            z[i] = dig + cin;
            p = dig == 0xffffffffu;
        } else {
            z[i] = dig - cin;
            p = dig == 0u;
        }
        cin = gg[u] | (p & cin);
    }
    if (threadIdx.x == 0) agg[blockIdx.x] = total;
}

// z[c] = low(a_c x) + high(a_(c-1) x), carries resolved; z[L] = final word.
__global__ void __launch_bounds__(kLinThreads) mulu32_k1(uint32_t* z, const uint32_t* a, size_t L, uint32_t x,
                                                         uint32_t* agg)
{
    const size_t i0 = (size_t)blockIdx.x * kLinWPC + (size_t)threadIdx.x * kLinIPT;
    uint32_t d[kLinIPT], gg[kLinIPT];
    uint32_t gp = kGPIdentity;
    uint32_t prev_hi = 0;
    if (i0 > 0 && i0 - 1 < L) prev_hi = (uint32_t)(((uint64_t)a[i0 - 1] * x) >> 32);
#pragma unroll
    for (int u = 0; u < kLinIPT; u++) {
        const size_t i = i0 + u;
        uint32_t g = 0, dig = 0;
        if (i < L) {
            const uint64_t pr = (uint64_t)a[i] * x;
            const uint64_t s = (uint64_t)(uint32_t)pr + prev_hi;
            dig = (uint32_t)s;
            g = (uint32_t)(s >> 32);
            prev_hi = (uint32_t)(pr >> 32);
        }
        d[u] = dig;
        gg[u] = g;
        if (i < L) gp = gp_combine(gp, g | ((uint32_t)(dig == 0xffffffffu) << 1));
    }
    uint32_t total;
    uint32_t cin = block_gp_scan(gp, &total) & 1u;
#pragma unroll
    for (int u = 0; u < kLinIPT; u++) {
        const size_t i = i0 + u;
        if (i >= L) break;
        z[i] = d[u] + cin;
        cin = gg[u] | ((uint32_t)(d[u] == 0xffffffffu) & cin);
    }
    if (threadIdx.x == 0) agg[blockIdx.x] = total;
}

__global__ void mulu32_final_kernel(uint32_t* z, const uint32_t* a, size_t L, uint32_t x, const uint32_t* fc)
{
    // word L = high half of the top product + the carry out of word L-1
    z[L] = (uint32_t)(((uint64_t)a[L - 1] * x) >> 32) + *fc;
}

static size_t run_scan_phases(uint32_t* z, size_t n, uint32_t* agg, size_t nctas, uint32_t* final_carry,
                              CarryMode mode, cudaStream_t s)
{
    carry_scan_aggregates(agg, nctas, final_carry, s);
    carry_ripple(z, n, kLinWPC, agg, nctas, mode, s);
    return nctas;
}

void lin_addsub(uint32_t* z, size_t TL, const WordView& a, const WordView& b, int64_t bot, bool sub,
                uint32_t* d_final, cudaStream_t s)
{
    if (TL == 0) {
        PIC_CUDA(cudaMemsetAsync(d_final, 0, sizeof(uint32_t), s));
        return;
    }
    const size_t nctas = (TL + kLinWPC - 1) / kLinWPC;
    DevBuf<uint32_t> agg(nctas, s);
    ProfScope ps(KC_LINEAR, 12.0 * (double)TL, s);
    addsub_k1<<<(unsigned)nctas, kLinThreads, 0, s>>>(z, TL, a, b, bot, sub ? kCarrySub : kCarryAdd, agg.get());
    PIC_CHECK_LAUNCH();
    count_launch();
    run_scan_phases(z, TL, agg.get(), nctas, d_final, sub ? kCarrySub : kCarryAdd, s);
}

void lin_mul_u32(uint32_t* z, const uint32_t* a, size_t L, uint32_t x, cudaStream_t s)
{
    const size_t nctas = (L + kLinWPC - 1) / kLinWPC;
    DevBuf<uint32_t> agg(nctas, s), fc(1, s);
    ProfScope ps(KC_LINEAR, 8.0 * (double)L, s);
    mulu32_k1<<<(unsigned)nctas, kLinThreads, 0, s>>>(z, a, L, x, agg.get());
    PIC_CHECK_LAUNCH();
    count_launch();
    run_scan_phases(z, L, agg.get(), nctas, fc.get(), kCarryAdd, s);
    mulu32_final_kernel<<<1, 1, 0, s>>>(z, a, L, x, fc.get());
    PIC_CHECK_LAUNCH();
    count_launch();
}

// ---- leading zeros / compare -------------------------------------------------
__global__ void top_nonzero_kernel(const uint32_t* z, size_t n, unsigned long long* out)
{
    // out = 1 + highest index with z[i] != 0 (0 if all zero); out preset to 0
    unsigned long long mine = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        if (z[i] != 0) mine = i + 1;
    mine = warp_max_u64(mine);
    if ((threadIdx.x & 31) == 0 && mine) atomicMax(out, mine);
}

size_t lin_top_nonzero(const uint32_t* z, size_t n, cudaStream_t s)
{
    if (n == 0) return 0;
    DevBuf<unsigned long long> d(1, s);
    PIC_CUDA(cudaMemsetAsync(d.get(), 0, sizeof(unsigned long long), s));
    top_nonzero_kernel<<<grid_for(n, 256), 256, 0, s>>>(z, n, d.get());
    PIC_CHECK_LAUNCH();
    count_launch();
    uint32_t h[2];
    read_words(h, (const uint32_t*)d.get(), 2, s);
    return (size_t)h[0] | ((size_t)h[1] << 32);
}

// Highest magnitude position where the two windows differ: atomicMax over
// (mag - lo + 1); 0 when equal over [lo, hi).
__global__ void ucmp_kernel(WordView a, WordView b, int64_t lo, int64_t hi, unsigned long long* out)
{
    const int64_t n = hi - lo;
    unsigned long long mine = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t mag = lo + i;
        if (word_at(a.T, a.exp, a.L, mag) != word_at(b.T, b.exp, b.L, mag)) mine = (unsigned long long)(i + 1);
    }
    mine = warp_max_u64(mine);
    if ((threadIdx.x & 31) == 0 && mine) atomicMax(out, mine);
}

int lin_ucmp(const WordView& a, const WordView& b, cudaStream_t s)
{
    // BigFloat::ucmp, BigFloat.cpp:123-147
    const int64_t magA = a.exp + a.L, magB = b.exp + b.L;
    if (magA > magB) return 1;
    if (magA < magB) return -1;
    const int64_t lo = a.exp < b.exp ? a.exp : b.exp;
    const int64_t hi = magA;
    if (hi <= lo) return 0;
    DevBuf<unsigned long long> d(1, s);
    PIC_CUDA(cudaMemsetAsync(d.get(), 0, sizeof(unsigned long long), s));
    ucmp_kernel<<<grid_for((size_t)(hi - lo), 256), 256, 0, s>>>(a, b, lo, hi, d.get());
    PIC_CHECK_LAUNCH();
    count_launch();
    uint32_t h[2];
    read_words(h, (const uint32_t*)d.get(), 2, s);
    const unsigned long long r = (unsigned long long)h[0] | ((unsigned long long)h[1] << 32);
    if (r == 0) return 0;
    const int64_t mag = lo + (int64_t)r - 1;
    uint32_t wa = 0, wb = 0;
    if (mag >= a.exp && mag < a.exp + a.L) read_words(&wa, a.T + (mag - a.exp), 1, s);
    if (mag >= b.exp && mag < b.exp + b.L) read_words(&wb, b.T + (mag - b.exp), 1, s);
    return wa < wb ? -1 : 1;
}

}  // namespace pic
