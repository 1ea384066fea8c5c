// FP64 FFT engine (see fft.cuh) and the FFT product with its rounding check.
#include <math.h>

#include <mutex>
#include <vector>

#include "carry.cuh"
#include "common.cuh"
#include "fft.cuh"
#include "mul.cuh"
#include "ntt.cuh"

namespace pic {

static constexpr int kFftInnerBits = 13;  // in-CTA sub-transforms up to 2^13 points
static constexpr int kFftK = 30;          // outer twiddle order 2^30
static constexpr int kFftS = 15;          // outer split e = hi * 2^15 + lo

struct FftTables {
    double2* inner = nullptr;  // exp(+2 pi i j / 2^13), j < 2^12
    double2* olo = nullptr;    // exp(+2 pi i j / 2^30), j < 2^15
    double2* ohi = nullptr;    // exp(+2 pi i j 2^15 / 2^30), j < 2^15
};

static std::once_flag g_fft_once;
static FftTables g_fft;

static double2* upload2(const std::vector<double2>& v)
{
    double2* d = nullptr;
    PIC_CUDA(raw_dev_alloc((void**)&d, v.size() * sizeof(double2)));
    PIC_CUDA(cudaMemcpy(d, v.data(), v.size() * sizeof(double2), cudaMemcpyHostToDevice));
    return d;
}

// Table entries are cos/sin of 2 pi j / 2^m evaluated directly per entry, as
// fft_ensure_table does (FFT.cpp:45-56), never by recurrence.
static const FftTables& fft_tables()
{
    std::call_once(g_fft_once, [] {
        const double two_pi = 6.283185307179586476925286766559;
        std::vector<double2> in((size_t)1 << (kFftInnerBits - 1));
        for (size_t j = 0; j < in.size(); j++) {
            const double a = two_pi * (double)j / (double)(1 << kFftInnerBits);
            in[j] = make_double2(cos(a), sin(a));
        }
        std::vector<double2> lo((size_t)1 << kFftS), hi((size_t)1 << (kFftK - kFftS));
        for (size_t j = 0; j < lo.size(); j++) {
            const double a = two_pi * (double)j / (double)(1u << kFftK);
            lo[j] = make_double2(cos(a), sin(a));
        }
        for (size_t j = 0; j < hi.size(); j++) {
            const double a = two_pi * (double)j / (double)(1u << (kFftK - kFftS));
            hi[j] = make_double2(cos(a), sin(a));
        }
        g_fft.inner = upload2(in);
        g_fft.olo = upload2(lo);
        g_fft.ohi = upload2(hi);
    });
    return g_fft;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b)  // a * conj(b)
{
    return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

template <int B, bool INV>
__device__ __forceinline__ void fft_group(double2 (&x)[1 << B], int j, int lst, const double2* __restrict__ tw)
{
    if (!INV) {
#pragma unroll
        for (int l = 0; l < B; l++) {
            const int hm = 1 << (B - 1 - l);
            const int shift = kFftInnerBits - (B - l) - lst;
#pragma unroll
            for (int m = 0; m < (1 << B); m++) {
                if (m & hm) continue;
                const int t = j + ((m & (hm - 1)) << lst);
                const double2 w = __ldg(tw + (t << shift));
                const double2 a = x[m], b = x[m + hm];
                x[m] = cadd(a, b);
                x[m + hm] = cmul(csub(a, b), w);
            }
        }
    } else {
#pragma unroll
        for (int l = B - 1; l >= 0; l--) {
            const int hm = 1 << (B - 1 - l);
            const int shift = kFftInnerBits - (B - l) - lst;
#pragma unroll
            for (int m = 0; m < (1 << B); m++) {
                if (m & hm) continue;
                const int t = j + ((m & (hm - 1)) << lst);
                const double2 w = __ldg(tw + (t << shift));
                const double2 a = x[m], b = cmulc(x[m + hm], w);
                x[m] = cadd(a, b);
                x[m + hm] = csub(a, b);
            }
        }
    }
}

template <int B, bool INV>
__device__ __forceinline__ void fft_run_group(double2* ptr, int base, int j, int lst, int es, const double2* tw)
{
    double2 x[1 << B];
#pragma unroll
    for (int m = 0; m < (1 << B); m++) x[m] = ptr[(size_t)(base + (m << lst)) * es];
    fft_group<B, INV>(x, j, lst, tw);
#pragma unroll
    for (int m = 0; m < (1 << B); m++) ptr[(size_t)(base + (m << lst)) * es] = x[m];
}

template <bool INV>
__device__ void cta_fft(double2* s, int logn, int nt, int es, int ts, bool tr_fast, const double2* tw)
{
    const int nfull = logn / 3, rem = logn % 3;
    const int nr = nfull + (rem ? 1 : 0);
    for (int ri = 0; ri < nr; ri++) {
        const int r = INV ? (nr - 1 - ri) : ri;
        const int b = (r < nfull) ? 3 : rem;
        const int lB = logn - 3 * r;
        const int lst = lB - b;
        const int lgpt = logn - b;
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
            double2* ptr = s + (size_t)tr * ts;
            if (b == 3) fft_run_group<3, INV>(ptr, base, j, lst, es, tw);
            else if (b == 2) fft_run_group<2, INV>(ptr, base, j, lst, es, tw);
            else fft_run_group<1, INV>(ptr, base, j, lst, es, tw);
        }
        __syncthreads();
    }
}

__device__ __forceinline__ double2 fft_outer_root(const double2* lo, const double2* hi, uint64_t e, int lM)
{
    const uint64_t E = e << (kFftK - lM);
    return cmul(__ldg(hi + (E >> kFftS)), __ldg(lo + (E & ((1u << kFftS) - 1))));
}

template <bool INV>
__global__ void __launch_bounds__(512) fft_rows_kernel(FftBatch B, int k, int lr, int rpc, const double2* tw)
{
    extern __shared__ double2 fsm[];
    const int n = 1 << lr;
    const size_t rows_per_tr = (size_t)1 << (k - lr);
    const size_t row0 = (size_t)blockIdx.x * rpc;
    for (int idx = threadIdx.x; idx < rpc * n; idx += blockDim.x) {
        const size_t row = row0 + idx / n;
        const size_t tr = row / rows_per_tr, rr = row % rows_per_tr;
        fsm[idx] = B.data[tr * B.stride + (rr << lr) + idx % n];
    }
    __syncthreads();
    cta_fft<INV>(fsm, lr, rpc, 1, n, false, tw);
    for (int idx = threadIdx.x; idx < rpc * n; idx += blockDim.x) {
        const size_t row = row0 + idx / n;
        const size_t tr = row / rows_per_tr, rr = row % rows_per_tr;
        B.data[tr * B.stride + (rr << lr) + idx % n] = fsm[idx];
    }
}

template <bool INV>
__global__ void __launch_bounds__(256) fft_cols_kernel(FftBatch B, int k, int lpre, int lc, int W,
                                                       const double2* tw, const double2* olo, const double2* ohi)
{
    extern __shared__ double2 fsm[];
    const int lM = k - lpre - lc;
    const size_t M = (size_t)1 << lM;
    const size_t tiles_per_block = M / W;
    const size_t ctas_per_tr = tiles_per_block << lpre;
    const size_t cta = blockIdx.x;
    const size_t tr = cta / ctas_per_tr;
    const size_t rem = cta % ctas_per_tr;
    const size_t ob = rem / tiles_per_block;
    const size_t c0 = (rem % tiles_per_block) * W;
    double2* base = B.data + tr * B.stride + (ob << (k - lpre)) + c0;
    const int N1 = 1 << lc;
    const int lblock = k - lpre;
    for (int idx = threadIdx.x; idx < N1 * W; idx += blockDim.x) {
        const int m = idx / W, w = idx % W;
        double2 v = base[((size_t)m << lM) + w];
        if (INV) {
            const uint64_t k1 = __brev((unsigned)m) >> (32 - lc);
            v = cmulc(v, fft_outer_root(olo, ohi, (c0 + w) * k1, lblock));
        }
        fsm[idx] = v;
    }
    __syncthreads();
    cta_fft<INV>(fsm, lc, W, W, 1, true, tw);
    for (int idx = threadIdx.x; idx < N1 * W; idx += blockDim.x) {
        const int m = idx / W, w = idx % W;
        double2 v = fsm[idx];
        if (!INV) {
            const uint64_t k1 = __brev((unsigned)m) >> (32 - lc);
            v = cmul(v, fft_outer_root(olo, ohi, (c0 + w) * k1, lblock));
        }
        base[((size_t)m << lM) + w] = v;
    }
}

static std::vector<int> fft_pass_bits(int k)
{
    std::vector<int> bits;
    if (k <= kFftInnerBits) {
        bits.push_back(k);
        return bits;
    }
    const int row = 11, colmax = 9;  // 16-byte points: half the NTT's tile
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

static void fft_launch_rows(bool inv, const FftBatch& b, int k, int lr, cudaStream_t s)
{
    const FftTables& T = fft_tables();
    const int n = 1 << lr;
    int rpc = 1;
    if (lr == k) {
        rpc = (1 << 10) / n;
        if (rpc < 1) rpc = 1;
        while (rpc > 1 && (b.count % rpc)) rpc >>= 1;
    }
    const size_t grid = ((size_t)b.count << (k - lr)) / rpc;
    ProfScope ps(KC_FFT_ROWS, 32.0 * (double)b.count * (double)((size_t)1 << k), s);
    const size_t smem = (size_t)rpc * n * sizeof(double2);
    int threads = (rpc * n) / 8;
    if (threads < 32) threads = 32;
    if (threads > 512) threads = 512;
    if (inv) {
        if (smem > 48 * 1024)
            PIC_CUDA(cudaFuncSetAttribute(fft_rows_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        fft_rows_kernel<true><<<(unsigned)grid, threads, smem, s>>>(b, k, lr, rpc, T.inner);
    } else {
        if (smem > 48 * 1024)
            PIC_CUDA(cudaFuncSetAttribute(fft_rows_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        fft_rows_kernel<false><<<(unsigned)grid, threads, smem, s>>>(b, k, lr, rpc, T.inner);
    }
    PIC_CHECK_LAUNCH();
    count_launch();
}

static void fft_launch_cols(bool inv, const FftBatch& b, int k, int lpre, int lc, cudaStream_t s)
{
    const FftTables& T = fft_tables();
    const int W = 4;
    const size_t M = (size_t)1 << (k - lpre - lc);
    const size_t grid = ((size_t)b.count * (M / W)) << lpre;
    const size_t smem = ((size_t)W << lc) * sizeof(double2);
    ProfScope ps(KC_FFT_COLS, 32.0 * (double)b.count * (double)((size_t)1 << k), s);
    if (inv) {
        if (smem > 48 * 1024)
            PIC_CUDA(cudaFuncSetAttribute(fft_cols_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        fft_cols_kernel<true><<<(unsigned)grid, 256, smem, s>>>(b, k, lpre, lc, W, T.inner, T.olo, T.ohi);
    } else {
        if (smem > 48 * 1024)
            PIC_CUDA(cudaFuncSetAttribute(fft_cols_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        fft_cols_kernel<false><<<(unsigned)grid, 256, smem, s>>>(b, k, lpre, lc, W, T.inner, T.olo, T.ohi);
    }
    PIC_CHECK_LAUNCH();
    count_launch();
}

void fft_forward_dif(const FftBatch& b, int k, cudaStream_t s)
{
    PIC_REQUIRE(k >= 1 && k <= kFftK, PIC_ERR_INVALID, "FFT length out of range");
    const std::vector<int> bits = fft_pass_bits(k);
    int lpre = 0;
    for (size_t i = 0; i + 1 < bits.size(); i++) {
        fft_launch_cols(false, b, k, lpre, bits[i], s);
        lpre += bits[i];
    }
    fft_launch_rows(false, b, k, bits.back(), s);
}

void fft_inverse_dit(const FftBatch& b, int k, cudaStream_t s)
{
    PIC_REQUIRE(k >= 1 && k <= kFftK, PIC_ERR_INVALID, "FFT length out of range");
    const std::vector<int> bits = fft_pass_bits(k);
    fft_launch_rows(true, b, k, bits.back(), s);
    int lpre = k - bits.back();
    for (int i = (int)bits.size() - 2; i >= 0; i--) {
        lpre -= bits[i];
        fft_launch_cols(true, b, k, lpre, bits[i], s);
    }
}

__global__ void fft_pointwise_kernel(double2* T, const double2* A, size_t n)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        T[i] = cmul(T[i], A[i]);
}

void fft_pointwise(double2* T, const double2* A, size_t n, cudaStream_t s)
{
    fft_pointwise_kernel<<<grid_for(n, 256), 256, 0, s>>>(T, A, n);
    PIC_CHECK_LAUNCH();
    count_launch();
}

// Worst-case rounding error of a length-2^k FFT convolution of b-bit pieces,
// after C. Percival, "Rapid multiplication modulo the sum and difference of
// highly composite numbers" (Math. Comp. 72, 2003), Theorem 5.1:
//   err <= N X Y [ (1+e)^(3k) (1+e sqrt5)^(3k+1) (1+beta)^(3k) - 1 ]
// with X = Y = 2^b - 1, e = 2^-53 and beta the twiddle error (2.5 e here: each
// outer twiddle is the rounded product of two rounded table entries).
double fft_error_bound(int k, int bits)
{
    const double e = ldexp(1.0, -53), beta = 2.5 * e;
    const double X = ldexp(1.0, bits) - 1.0;
    const double lg = 3.0 * k * log1p(e) + (3.0 * k + 1) * log1p(e * sqrt(5.0)) + 3.0 * k * log1p(beta);
    return ldexp(1.0, k) * X * X * expm1(lg);
}

int fft_piece_bits(int k)
{
    for (int b = 16; b >= 8; b--)
        if (fft_error_bound(k, b) < 0.25) return b;
    return 0;
}

__global__ void fft_split_kernel(double2* T, size_t N, const uint32_t* A, size_t AL, int bits)
{
    const uint32_t mask = (1u << bits) - 1u;
    const size_t nbits = AL * 32;
    for (size_t j = blockIdx.x * (size_t)blockDim.x + threadIdx.x; j < N; j += (size_t)gridDim.x * blockDim.x) {
        double v = 0;
        const size_t b0 = j * (size_t)bits;
        if (b0 < nbits) {
            const size_t w = b0 >> 5;
            const int r = (int)(b0 & 31);
            uint64_t x = A[w];
            if (w + 1 < AL) x |= (uint64_t)A[w + 1] << 32;
            v = (double)((uint32_t)(x >> r) & mask);
        }
        T[j] = make_double2(v, 0.0);
    }
}

void fft_split(double2* T, int k, const uint32_t* A, size_t AL, int bits, cudaStream_t s)
{
    const size_t N = (size_t)1 << k;
    fft_split_kernel<<<grid_for(N, 256), 256, 0, s>>>(T, N, A, AL, bits);
    PIC_CHECK_LAUNCH();
    count_launch();
}

bool mul_fft(uint32_t* z, const uint32_t* a, size_t na, const uint32_t* b, size_t nb, cudaStream_t s,
             double* max_err)
{
    const size_t zw = na + nb;
    int k = 1, bits = 0;
    for (k = 1; k <= kFftK; k++) {
        const int bb = fft_piece_bits(k);
        if (bb == 0) break;
        if (((size_t)1 << k) * (size_t)bb >= 32 * zw) {
            bits = bb;
            break;
        }
    }
    PIC_REQUIRE(bits != 0, PIC_ERR_LENGTH, "product too long for a provably exact FP64 FFT");
    const size_t N = (size_t)1 << k;
    const bool square = (a == b && na == nb);
    DevBuf<double2> A(N, s), B(square ? 0 : N, s);
    fft_split(A.get(), k, a, na, bits, s);
    fft_forward_dif(FftBatch{A.get(), N, 1}, k, s);
    if (!square) {
        fft_split(B.get(), k, b, nb, bits, s);
        fft_forward_dif(FftBatch{B.get(), N, 1}, k, s);
    }
    fft_pointwise(A.get(), square ? A.get() : B.get(), N, s);
    fft_inverse_dit(FftBatch{A.get(), N, 1}, k, s);
    const size_t ncoef = (32 * zw + bits - 1) / bits;
    const double err = fft_coef_to_words(A.get(), ncoef < N ? ncoef : N, 1.0 / (double)N, bits, z, zw, s);
    fft_note_max_err(err);
    if (max_err) *max_err = err;
    return err <= 0.25;
}

}  // namespace pic
