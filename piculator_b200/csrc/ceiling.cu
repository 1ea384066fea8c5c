// The integer roofline of the NTT passes: the rate of lazy Shoup DIF
// butterflies (the arithmetic of ntt_rows_fast_kernel / ntt_cols_fast_kernel,
// mod the first product prime: operands in [0, 4p), three-partial-product
// quotient) with operands and twiddles in registers, no memory traffic.  Radix-8 groups, 12 butterflies per group, 8 resident CTAs
// of 256 threads per SM.
#include <string.h>

#include "common.cuh"
#include "fp64mod.cuh"
#include "modarith.cuh"
#include "ntt.cuh"

namespace pic {

__global__ void __launch_bounds__(256) butterfly_ceiling_kernel(uint64_t* out, const uint64_t* tw, uint64_t p,
                                                                int iters)
{
    const uint32_t c = (uint32_t)(p >> 32);
    const uint64_t p4 = 4 * p;
    uint64_t x[8];
    for (int m = 0; m < 8; m++) x[m] = (threadIdx.x * 8 + m + blockIdx.x) % p;
    uint64_t w[7], ws[7];
    for (int i = 0; i < 7; i++) {
        w[i] = tw[2 * (i + threadIdx.x % 8)];
        ws[i] = tw[2 * (i + threadIdx.x % 8) + 1];
    }
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int l = 0; l < 3; l++) {
            const int hm = 4 >> l;
#pragma unroll
            for (int m = 0; m < 8; m++) {
                if (m & hm) continue;
                const int ti = (l == 0 ? 0 : (l == 1 ? 4 : 6)) + (m & (hm - 1));
                uint64_t s = x[m] + x[m + hm];
                s = s >= p4 ? s - p4 : s;
                x[m + hm] = shoup_approx32(x[m] + p4 - x[m + hm], w[ti], ws[ti], c);
                x[m] = s;
            }
        }
    }
    uint64_t acc = 0;
    for (int m = 0; m < 8; m++) acc ^= x[m];
    out[blockIdx.x * (size_t)blockDim.x + threadIdx.x] = acc;
}

// The same radix-8 DIF groups with the FP64 butterflies of the FP64 form
// (fp64mod.cuh, twiddles w with the companion formed per use): signed
// residues below p in and out of every group, the sums reduced at the
// group's last level, mod the first FP64 prime.
__global__ void __launch_bounds__(256) butterfly_ceiling_dbl_kernel(uint64_t* out, const uint64_t* tw, double p,
                                                                    int iters)
{
    const double pinv = 1.0 / p;
    double x[8];
    for (int m = 0; m < 8; m++) x[m] = dreduce((double)(threadIdx.x * 8 + m + blockIdx.x), p, pinv);
    double w[7];
    for (int i = 0; i < 7; i++) w[i] = dbits(tw[i + threadIdx.x % 8]);
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int l = 0; l < 3; l++) {
            const int hm = 4 >> l;
#pragma unroll
            for (int m = 0; m < 8; m++) {
                if (m & hm) continue;
                const int ti = (l == 0 ? 0 : (l == 1 ? 4 : 6)) + (m & (hm - 1));
                const double sm = __dadd_rn(x[m], x[m + hm]), d = __dadd_rn(x[m], -x[m + hm]);
                x[m + hm] = dmul_w(d, w[ti], p, pinv);
                x[m] = l == 2 ? dreduce(sm, p, pinv) : sm;
            }
        }
    }
    double acc = 0;
    for (int m = 0; m < 8; m++) acc += x[m];
    out[blockIdx.x * (size_t)blockDim.x + threadIdx.x] = dstore(acc);
}

double butterfly_ceiling_dbl(cudaStream_t s)
{
    const uint64_t p = kDblPrimes[0];
    uint64_t htw[32];
    uint64_t w = 1;
    const uint64_t g = host_powmod(smallest_generator(p), (p - 1) >> 16, p);  // a root of order 2^16
    for (int i = 0; i < 32; i++) {
        const double wd = (double)w;
        memcpy(&htw[i], &wd, 8);
        w = host_mulmod(w, g, p);
    }
    const int blocks = ctx().num_sms * 8, threads = 256, iters = 1000;
    DevBuf<uint64_t> dtw(32, s), dout((size_t)blocks * threads, s);
    PIC_CUDA(cudaMemcpyAsync(dtw.get(), htw, sizeof htw, cudaMemcpyHostToDevice, s));
    cudaEvent_t e0, e1;
    PIC_CUDA(cudaEventCreate(&e0));
    PIC_CUDA(cudaEventCreate(&e1));
    float best = 0.f;
    for (int rep = 0; rep < 3; rep++) {
        PIC_CUDA(cudaEventRecord(e0, s));
        butterfly_ceiling_dbl_kernel<<<blocks, threads, 0, s>>>(dout.get(), dtw.get(), (double)p, iters);
        PIC_CHECK_LAUNCH();
        count_launch();
        PIC_CUDA(cudaEventRecord(e1, s));
        PIC_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        PIC_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (rep > 0 && (best == 0.f || ms < best)) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const double bfly = (double)blocks * threads * iters * 12.0;
    return bfly / (best * 1e-3) / 1e9;  // G butterflies / s
}

double butterfly_ceiling(cudaStream_t s)
{
    const uint64_t p = kProductPrimes[0];
    uint64_t htw[32];
    uint64_t w = 1;
    const uint64_t g = host_powmod(smallest_generator(p), (p - 1) >> 16, p);  // a root of order 2^16
    for (int i = 0; i < 16; i++) {
        htw[2 * i] = w;
        htw[2 * i + 1] = shoup_companion(w, p);
        w = host_mulmod(w, g, p);
    }
    const int blocks = ctx().num_sms * 8, threads = 256, iters = 1000;
    DevBuf<uint64_t> dtw(32, s), dout((size_t)blocks * threads, s);
    PIC_CUDA(cudaMemcpyAsync(dtw.get(), htw, sizeof htw, cudaMemcpyHostToDevice, s));
    cudaEvent_t e0, e1;
    PIC_CUDA(cudaEventCreate(&e0));
    PIC_CUDA(cudaEventCreate(&e1));
    float best = 0.f;
    for (int rep = 0; rep < 3; rep++) {
        PIC_CUDA(cudaEventRecord(e0, s));
        butterfly_ceiling_kernel<<<blocks, threads, 0, s>>>(dout.get(), dtw.get(), p, iters);
        PIC_CHECK_LAUNCH();
        count_launch();
        PIC_CUDA(cudaEventRecord(e1, s));
        PIC_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        PIC_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (rep > 0 && (best == 0.f || ms < best)) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const double bfly = (double)blocks * threads * iters * 12.0;
    return bfly / (best * 1e-3) / 1e9;  // G butterflies / s
}

}  // namespace pic
