// BigFloat linear kernels: windowed add/subtract (uadd/usub, BigFloat.cpp:
// 184-287), multiply by a 32-bit word (BigFloat.cpp:156-183), leading-zero
// strip and magnitude compare (BigFloat.cpp:123-147).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pic {

// A magnitude as the reference stores it: words T[0..L) at exponent exp.
struct WordView {
    const uint32_t* T;
    int64_t exp;
    int64_t L;
};

// z[0..TL) = a(bot + c) +/- b(bot + c) with carries/borrows; *d_final (device)
// receives the carry (add) or borrow (subtract) out of word TL-1.
void lin_addsub(uint32_t* z, size_t TL, const WordView& a, const WordView& b, int64_t bot, bool sub,
                uint32_t* d_final, cudaStream_t s);
// z[0..L] = a[0..L) * x (z has L+1 words; z[L] may be 0).
void lin_mul_u32(uint32_t* z, const uint32_t* a, size_t L, uint32_t x, cudaStream_t s);
// 1 + index of the highest nonzero word (0 if none).  Synchronises.
size_t lin_top_nonzero(const uint32_t* z, size_t n, cudaStream_t s);
// Sign of |a| - |b| over aligned magnitudes.  Synchronises.
int lin_ucmp(const WordView& a, const WordView& b, cudaStream_t s);

}  // namespace pic
