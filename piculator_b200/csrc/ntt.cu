// NTT engine kernels and twiddle tables (see ntt.cuh for the layout).
#include <stdio.h>
#include <string.h>

#include <map>
#include <mutex>

#include "common.cuh"
#include "ntt.cuh"

namespace pic {

// Three primes c * 2^32 + 1 below 2^62 (2-adicity 33, 34, 37); their product
// is ~2^186, so a cyclic convolution of 64-bit pieces of length <= 2^30 (any
// coefficient < 2^158, or a signed difference of two such) is recovered
// exactly by CRT.
const uint64_t kProductPrimes[3] = {4611685941117976577ull, 4611685692009873409ull,
                                    4611685606110527489ull};

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
    PIC_CUDA(cudaMalloc(&d, v.size() * sizeof(uint64_t)));
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
    d.inner_fwd = upload(inf);
    d.inner_inv = upload(ini);
    d.olo_fwd = upload(lof);
    d.ohi_fwd = upload(hif);
    d.olo_inv = upload(loi);
    d.ohi_inv = upload(hii);
    g_tabs[p] = t;
    return *t;
}

std::vector<int> ntt_pass_bits(int k)
{
    std::vector<int> bits;
    if (k <= kInnerBits) {
        bits.push_back(k);
        return bits;
    }
    const int row = 12, colmax = 10;
    int rest = k - row;
    int ncol = (rest + colmax - 1) / colmax;
    for (int i = 0; i < ncol; i++) {
        int b = rest / (ncol - i) + ((rest % (ncol - i)) ? 1 : 0);
        bits.push_back(b);
        rest -= b;
    }
    bits.push_back(row);
    return bits;
}

// ---------------------------------------------------------------------------
// In-CTA transform: radix-2^B register groups, shared-memory exchanges.

// One group of 2^B elements at positions base + j + m * 2^lst of a sub-block
// of size 2^(lst + B); performs the B butterfly levels of that sub-block.
template <int B, bool INV>
__device__ __forceinline__ void group_levels(uint64_t (&x)[1 << B], int j, int lst, const PrimeDev& P)
{
    const uint64_t p = P.p;
    const uint64_t* __restrict__ tw = INV ? P.inner_inv : P.inner_fwd;
    if (!INV) {
#pragma unroll
        for (int l = 0; l < B; l++) {
            const int hm = 1 << (B - 1 - l);
            const int shift = P.IB - (B - l) - lst;  // root of order 2h = 2^(B-l+lst)
#pragma unroll
            for (int m = 0; m < (1 << B); m++) {
                if (m & hm) continue;
                const int t = j + ((m & (hm - 1)) << lst);
                const int ti = t << shift;
                const uint64_t w = __ldg(tw + 2 * ti), ws = __ldg(tw + 2 * ti + 1);
                const uint64_t a = x[m], b = x[m + hm];
                x[m] = add_mod(a, b, p);
                x[m + hm] = shoup_mul(sub_mod(a, b, p), w, ws, p);
            }
        }
    } else {
#pragma unroll
        for (int l = B - 1; l >= 0; l--) {
            const int hm = 1 << (B - 1 - l);
            const int shift = P.IB - (B - l) - lst;
#pragma unroll
            for (int m = 0; m < (1 << B); m++) {
                if (m & hm) continue;
                const int t = j + ((m & (hm - 1)) << lst);
                const int ti = t << shift;
                const uint64_t w = __ldg(tw + 2 * ti), ws = __ldg(tw + 2 * ti + 1);
                const uint64_t a = x[m], b = shoup_mul(x[m + hm], w, ws, p);
                x[m] = add_mod(a, b, p);
                x[m + hm] = sub_mod(a, b, p);
            }
        }
    }
}

template <int B, bool INV>
__device__ __forceinline__ void run_group(uint64_t* __restrict__ ptr, int base, int j, int lst, int es,
                                          const PrimeDev& P)
{
    uint64_t x[1 << B];
#pragma unroll
    for (int m = 0; m < (1 << B); m++) x[m] = ptr[(size_t)(base + (m << lst)) * es];
    group_levels<B, INV>(x, j, lst, P);
#pragma unroll
    for (int m = 0; m < (1 << B); m++) ptr[(size_t)(base + (m << lst)) * es] = x[m];
}

// nt transforms of size 2^logn in shared memory; element m of transform t
// lives at s[t * ts + m * es].  tr_fast picks which index consecutive threads
// walk (transforms for column tiles, elements for rows).
template <bool INV>
__device__ void cta_ntt(uint64_t* s, int logn, int nt, int es, int ts, bool tr_fast, const PrimeDev& P)
{
    const int nfull = logn / 3, rem = logn % 3;
    const int nr = nfull + (rem ? 1 : 0);
    for (int ri = 0; ri < nr; ri++) {
        const int r = INV ? (nr - 1 - ri) : ri;
        const int b = (r < nfull) ? 3 : rem;
        const int lB = logn - 3 * r;  // log2 sub-block size
        const int lst = lB - b;       // log2 stride inside the group
        const int lgpt = logn - b;    // log2 groups per transform
        const int G = nt << lgpt;
        for (int g = threadIdx.x; g < G; g += blockDim.x) {
            int tr, gi;
            if (tr_fast) {
                tr = g % nt;
                gi = g / nt;
            } else {
                tr = g >> lgpt;
                gi = g & ((1 << lgpt) - 1);
            }
            const int sb = gi >> lst, j = gi & ((1 << lst) - 1);
            const int base = (sb << lB) + j;
            uint64_t* ptr = s + (size_t)tr * ts;
            if (b == 3) run_group<3, INV>(ptr, base, j, lst, es, P);
            else if (b == 2) run_group<2, INV>(ptr, base, j, lst, es, P);
            else run_group<1, INV>(ptr, base, j, lst, es, P);
        }
        __syncthreads();
    }
}

__device__ __forceinline__ const PrimeDev& prime_of(const NttBatch& B, int i)
{
    int q = i / B.per_prime;
    return B.prime[q];
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

// Contiguous row pass: rows of 2^lr elements; rpc rows per CTA.
template <bool INV>
__global__ void __launch_bounds__(512) ntt_rows_kernel(NttBatch B, int k, int lr, int rpc)
{
    extern __shared__ uint64_t smem[];
    const int n = 1 << lr;
    const size_t rows_per_tr = (size_t)1 << (k - lr);
    const size_t row0 = (size_t)blockIdx.x * rpc;
    const int tr0 = (int)(row0 / rows_per_tr);
    const PrimeDev& P = prime_of(B, tr0);
    // load rpc rows (contiguous when rows belong to the same transform)
    for (int idx = threadIdx.x; idx < rpc * n; idx += blockDim.x) {
        const size_t row = row0 + idx / n;
        const int e = idx % n;
        const size_t tr = row / rows_per_tr, rr = row % rows_per_tr;
        smem[idx] = B.data[tr * B.stride + (rr << lr) + e];
    }
    __syncthreads();
    cta_ntt<INV>(smem, lr, rpc, 1, n, false, P);
    for (int idx = threadIdx.x; idx < rpc * n; idx += blockDim.x) {
        const size_t row = row0 + idx / n;
        const int e = idx % n;
        const size_t tr = row / rows_per_tr, rr = row % rows_per_tr;
        B.data[tr * B.stride + (rr << lr) + e] = smem[idx];
    }
}

// Strided column pass.  The transform is a sequence of 2^lpre outer blocks of
// 2^(k-lpre) elements; each outer block is an N1 x M tile (N1 = 2^lc rows,
// M = 2^(k-lpre-lc) columns, row-major).  A CTA owns W columns of one tile.
template <bool INV>
__global__ void __launch_bounds__(256) ntt_cols_kernel(NttBatch B, int k, int lpre, int lc, int W)
{
    extern __shared__ uint64_t smem[];
    const int lM = k - lpre - lc;
    const size_t M = (size_t)1 << lM;
    const size_t tiles_per_block = M / W;
    const size_t ctas_per_tr = tiles_per_block << lpre;
    const size_t cta = blockIdx.x;
    const int tr = (int)(cta / ctas_per_tr);
    const size_t rem = cta % ctas_per_tr;
    const size_t ob = rem / tiles_per_block;
    const size_t c0 = (rem % tiles_per_block) * W;
    const PrimeDev& P = prime_of(B, tr);
    uint64_t* base = B.data + (size_t)tr * B.stride + (ob << (k - lpre)) + c0;
    const int N1 = 1 << lc;
    const int lblock = k - lpre;  // twiddle root order 2^lblock

    for (int idx = threadIdx.x; idx < N1 * W; idx += blockDim.x) {
        const int m = idx / W, w = idx % W;
        uint64_t v = base[((size_t)m << lM) + w];
        if (INV) {
            const uint64_t k1 = __brev((unsigned)m) >> (32 - lc);
            v = mont_mul(v, outer_root<true>(P, (c0 + w) * k1, lblock), P.p, P.pinv_neg);
        }
        smem[idx] = v;
    }
    __syncthreads();
    cta_ntt<INV>(smem, lc, W, W, 1, true, P);
    for (int idx = threadIdx.x; idx < N1 * W; idx += blockDim.x) {
        const int m = idx / W, w = idx % W;
        uint64_t v = smem[idx];
        if (!INV) {
            const uint64_t k1 = __brev((unsigned)m) >> (32 - lc);
            v = mont_mul(v, outer_root<false>(P, (c0 + w) * k1, lblock), P.p, P.pinv_neg);
        }
        base[((size_t)m << lM) + w] = v;
    }
}

static constexpr int kColW = 8;

static void launch_rows(bool inv, const NttBatch& b, int k, int lr, cudaStream_t s)
{
    const int n = 1 << lr;
    int rpc = 1;
    if (lr == k) {
        // several whole transforms per CTA when short, never straddling primes
        rpc = (1 << 11) / n;
        if (rpc < 1) rpc = 1;
        while (rpc > 1 && (b.per_prime % rpc)) rpc >>= 1;
    }
    const size_t rows = (size_t)b.count << (k - lr);
    const size_t grid = rows / rpc;
    ProfScope ps(KC_NTT_ROWS, 16.0 * (double)b.count * (double)((size_t)1 << k), s);
    const size_t smem = (size_t)rpc * n * sizeof(uint64_t);
    int threads = (rpc * n) / 8;
    if (threads < 32) threads = 32;
    if (threads > 512) threads = 512;
    if (inv) {
        if (smem > 48 * 1024)
            PIC_CUDA(cudaFuncSetAttribute(ntt_rows_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        ntt_rows_kernel<true><<<(unsigned)grid, threads, smem, s>>>(b, k, lr, rpc);
    } else {
        if (smem > 48 * 1024)
            PIC_CUDA(cudaFuncSetAttribute(ntt_rows_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        ntt_rows_kernel<false><<<(unsigned)grid, threads, smem, s>>>(b, k, lr, rpc);
    }
    PIC_CHECK_LAUNCH();
    count_launch();
}

static void launch_cols(bool inv, const NttBatch& b, int k, int lpre, int lc, cudaStream_t s)
{
    const int W = kColW;
    const size_t M = (size_t)1 << (k - lpre - lc);
    const size_t grid = (size_t)b.count * (M / W) << lpre;
    const size_t smem = ((size_t)W << lc) * sizeof(uint64_t);
    ProfScope ps(KC_NTT_COLS, 16.0 * (double)b.count * (double)((size_t)1 << k), s);
    if (inv) {
        if (smem > 48 * 1024)
            PIC_CUDA(cudaFuncSetAttribute(ntt_cols_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        ntt_cols_kernel<true><<<(unsigned)grid, 256, smem, s>>>(b, k, lpre, lc, W);
    } else {
        if (smem > 48 * 1024)
            PIC_CUDA(cudaFuncSetAttribute(ntt_cols_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        ntt_cols_kernel<false><<<(unsigned)grid, 256, smem, s>>>(b, k, lpre, lc, W);
    }
    PIC_CHECK_LAUNCH();
    count_launch();
}

static void check_batch(const NttBatch& b, int k)
{
    PIC_REQUIRE(k >= 1 && k <= 32, PIC_ERR_INVALID, "NTT length out of range");
    PIC_REQUIRE(b.count > 0 && b.per_prime > 0 && b.count <= b.per_prime * kMaxPrimesPerBatch,
                PIC_ERR_INVALID, "bad NTT batch");
    PIC_REQUIRE(b.stride >= ((size_t)1 << k), PIC_ERR_INVALID, "NTT batch stride too small");
    for (int q = 0; q * b.per_prime < b.count; q++)
        PIC_REQUIRE(b.prime[q].K >= k, PIC_ERR_INVALID, "prime has no root of unity of this order");
}

void ntt_forward_dif(const NttBatch& b, int k, cudaStream_t s)
{
    check_batch(b, k);
    std::vector<int> bits = ntt_pass_bits(k);
    int lpre = 0;
    for (size_t i = 0; i + 1 < bits.size(); i++) {
        launch_cols(false, b, k, lpre, bits[i], s);
        lpre += bits[i];
    }
    launch_rows(false, b, k, bits.back(), s);
}

void ntt_inverse_dit(const NttBatch& b, int k, cudaStream_t s)
{
    check_batch(b, k);
    std::vector<int> bits = ntt_pass_bits(k);
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

__global__ void pointwise_mont_kernel(NttBatch B, const uint64_t* __restrict__ other, int k)
{
    const size_t n = (size_t)1 << k;
    const size_t total = (size_t)B.count * n;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < total;
         g += (size_t)gridDim.x * blockDim.x) {
        const size_t tr = g >> k, i = g & (n - 1);
        const PrimeDev& P = prime_of(B, (int)tr);
        uint64_t* d = B.data + tr * B.stride + i;
        *d = mont_mul(*d, other[tr * B.stride + i], P.p, P.pinv_neg);
    }
}

void ntt_pointwise_mont(const NttBatch& a, const uint64_t* b, int k, cudaStream_t s)
{
    const size_t total = (size_t)a.count << k;
    ProfScope ps(KC_NTT_POINTWISE, 24.0 * (double)total, s);
    pointwise_mont_kernel<<<grid_for(total, 256), 256, 0, s>>>(a, b, k);
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
