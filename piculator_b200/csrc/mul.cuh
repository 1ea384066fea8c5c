// Exact big-integer products on the device (the inner product of
// BigFloat::mul, BigFloat.cpp:413-487): z[0 .. na+nb) = a * b.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ntt.cuh"
#include "piculator_b200.h"

namespace pic {

// Three-prime NTT: 64-bit pieces, primes kProductPrimes, Garner CRT.
void mul_ntt3(uint32_t* z, const uint32_t* a, size_t na, const uint32_t* b, size_t nb, cudaStream_t s);
// The same in FP64 arithmetic: 56-bit pieces, primes kDblPrimes (fp64mod.cuh).
void mul_ntt3d(uint32_t* z, const uint32_t* a, size_t na, const uint32_t* b, size_t nb, cudaStream_t s);
// 56-bit pieces of an operand of n words.
size_t pieces56(size_t nwords);
// FP64-form building blocks: split + forward into out[3 * 2^k]; batched
// inverse output like ntt3_batch_to_words (offset 2^140 per coefficient);
// wrapped-product fix-up like launch_wrap_fix.
void ntt3d_forward_operand(uint64_t* out, int k, const uint32_t* a, size_t na, cudaStream_t s);
void ntt3d_batch_to_words(const uint64_t* y, size_t istride, size_t pstride, size_t count, int k, uint32_t* z,
                          uint32_t zcap, const uint32_t* zlen, cudaStream_t s, size_t ncoef, bool offset);
void launch_wrap_fix_d(uint64_t* y, size_t ystride, const uint64_t* tail, size_t T, size_t nitems,
                       size_t item_mul, size_t nchild, size_t Nm, size_t W, cudaStream_t s);
// The three-prime form of AUTO products and binary-splitting merges
// (kFormInt, kFormDbl, or kFormChosen: per product by transform work).
void mul_set_ntt_form(int form);
int mul_ntt_form();
// The form a product of operands of the given piece counts (64-bit pieces
// for the integer form, 56-bit for the FP64 one) takes under the setting.
int ntt_form_for(size_t pieces_int_a, size_t pieces_int_b, size_t pieces_dbl_a, size_t pieces_dbl_b, bool wrap);

// While alive, three-prime products on this thread that take the operand
// (src, n) transform it once per transform length and reuse that forward
// transform (the Newton steps multiply by their iterate twice,
// BigFloat.cpp:510, 561-567).  Scopes nest.
class OperandHold {
public:
    OperandHold(const uint32_t* src, size_t n);
    ~OperandHold();
    OperandHold(const OperandHold&) = delete;
    OperandHold& operator=(const OperandHold&) = delete;

private:
    void* prev_;
    void* held_;
};
// Products that found the held transform ready (since the process started).
uint64_t held_transform_reuses();
// The reference's own layout: 16-bit points in u64, one prime (the
// reference's prime for k), length 2^k >= 4 (na + nb) (BigFloat.cpp:380-385).
void mul_ntt_ref(uint32_t* z, const uint32_t* a, size_t na, const uint32_t* b, size_t nb, cudaStream_t s);
// One CTA per product, column sums in shared memory (na + nb <= kSchoolMax).
constexpr size_t kSchoolMaxWords = 4096;
void mul_school(uint32_t* z, const uint32_t* a, size_t na, const uint32_t* b, size_t nb, cudaStream_t s);
// FP64 FFT product; returns false (and leaves z undefined) when the largest
// rounding distance exceeded 0.25, so the caller can recompute exactly.
bool mul_fft(uint32_t* z, const uint32_t* a, size_t na, const uint32_t* b, size_t nb, cudaStream_t s,
             double* max_err);

// Three-prime building blocks (also used by transform-domain operands):
// split + forward into out[3 * 2^k]; pointwise a *= b (adds one R^-1);
// inverse + CRT + carry of coefficients [0, ncoef) into zw words, undoing
// `depth` Montgomery factors.
void ntt3_forward_operand(uint64_t* out, int k, const uint32_t* a, size_t na, cudaStream_t s);
void ntt3_pointwise(uint64_t* a, const uint64_t* b, int k, cudaStream_t s);
void ntt3_inverse_to_words(uint64_t* y, int k, size_t ncoef, int depth, uint32_t* z, size_t zw, cudaStream_t s);

// Batched inverse output: product i's residues at y + i * istride + q * pstride
// (transform length 2^k, already inverse-transformed, one pointwise Montgomery
// factor); zlen[i] words into z + i * zcap.  ncoef (default 2^k) is the number
// of coefficients read per product: a wrapped product stores its top
// coefficients past the transform, at indices 2^k .. ncoef - 1.
// Wrapped form of the three-prime product in mul_ntt3 (on by default).
void mul_set_wrap(bool on);
bool mul_wrap();

// Wrapped products (see wrap_fix_kernel in mul.cu): nitems products, item
// it of prime q at y + (q nchild + it item_mul) ystride (main, length Nm) and
// tail + (q nchild + it item_mul) T (tail product, length T); cT = Nm / T in
// Montgomery form per prime.
void launch_wrap_fix(uint64_t* y, size_t ystride, const uint64_t* tail, size_t T, size_t nitems, size_t item_mul,
                     size_t nchild, size_t Nm, size_t W, const uint64_t cT[3], cudaStream_t s);

// With `offset`, every coefficient j < ncoef is converted as c_j + 2^159 (for
// signed coefficients |c_j| < 2^159): the words are the value plus the fixed
// integer sum_j 2^(159 + 64 j).
void ntt3_batch_to_words(const uint64_t* y, size_t istride, size_t pstride, size_t count, int k, uint32_t* z,
                         uint32_t zcap, const uint32_t* zlen, cudaStream_t s, size_t ncoef = 0, bool offset = false);

// batch.cu: persistent schoolbook + binned three-prime NTT, replayed from a
// CUDA graph when the sizes repeat.
void mul_batch(const pic_mul_desc* d, size_t count, int mode, cudaStream_t s);
void mul_batch_set_graphs(bool on);
// noalloc.cu: the three-prime product in fixed library storage (no allocation).
void mul_noalloc(uint32_t* z, const uint32_t* a, size_t na, const uint32_t* b, size_t nb, cudaStream_t s);

// Caller-supplied-buffer forms of the three-prime pieces (noalloc.cu):
// split3_into writes 3 * 2^k residues mod primes[0..2]; crt3_to_words_scratch
// needs crt3_scratch_ctas(zw) words of `agg` and ncoef <= 2^k.
void split3_into(uint64_t* out, int k, const uint32_t* a, size_t na, const uint64_t primes[3], cudaStream_t s);
size_t crt3_scratch_ctas(size_t zw);
void crt3_to_words_scratch(const uint64_t* y, int k, size_t ncoef, uint32_t* z, size_t zw, uint32_t* agg,
                           cudaStream_t s);

// Dispatch on mode (PIC_MUL_*).
void mul_dispatch(uint32_t* z, const uint32_t* a, size_t na, const uint32_t* b, size_t nb, int mode,
                  cudaStream_t s);
int mul_auto_mode(size_t na, size_t nb);
void mul_set_thresholds(int64_t school_max, int64_t fft_max);
int64_t mul_school_max();
int64_t mul_fft_max();

// Reference-API conversions (NTT.cpp:330-369).
void int_to_ntt_dev(uint64_t* T, int k, const uint32_t* A, size_t AL, cudaStream_t s);
void ntt_to_int_dev(const uint64_t* T, int k, uint32_t* A, size_t AL, cudaStream_t s);

// Coefficients (already reduced, one prime, 16-bit positions) -> words, with
// optional Montgomery rescale; shared by ntt_to_int_dev and mul_ntt_ref.
void coef16_to_words(const uint64_t* c, size_t ncoef, uint64_t scale_mont, uint64_t p, uint64_t pinv_neg,
                     uint32_t* z, size_t zw, cudaStream_t s);

// FFT coefficients (real parts times scale, rounded) at b-bit positions ->
// words; returns the largest rounding distance seen.  Synchronises.
double fft_coef_to_words(const double2* T, size_t ncoef, double scale, int bits, uint32_t* z, size_t zw,
                         cudaStream_t s);

double fft_last_max_err();
void fft_note_max_err(double e);
// Largest FFT rounding distance noted since the last reset (pi statistics).
double fft_max_err_seen();
void fft_reset_max_err();
// FFT acceptance threshold (max distance to the nearest integer; default 0.25).
void mul_set_fft_accept(double max_dist);
double mul_fft_accept();

}  // namespace pic
