// FP64 complex FFT with the reference's conventions (FFT.cpp:31-463):
// forward = DIF, twiddles exp(+2 pi i t / 2h), natural in, bit-reversed out;
// inverse = DIT, conjugate twiddles, bit-reversed in, natural out, unscaled.
// Same pass structure as the NTT engine (ntt.cuh): strided column passes with
// the inter-step twiddle, one contiguous row pass, radix-8 register groups.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pic {

struct FftBatch {
    double2* data;
    size_t stride;  // complex elements between transforms
    int count;
};

void fft_forward_dif(const FftBatch& b, int k, cudaStream_t s);
void fft_inverse_dit(const FftBatch& b, int k, cudaStream_t s);
void fft_pointwise(double2* T, const double2* A, size_t n, cudaStream_t s);

// Largest piece width b (bits) whose worst-case rounding error for a length
// 2^k product of b-bit pieces stays below 1/4 (error bound in fft.cu); 0 if
// even 8-bit pieces are not provably safe at this length.
int fft_piece_bits(int k);
double fft_error_bound(int k, int bits);

// Splits words into b-bit pieces (real part), zero-padded to 2^k points.
void fft_split(double2* T, int k, const uint32_t* A, size_t AL, int bits, cudaStream_t s);

}  // namespace pic
