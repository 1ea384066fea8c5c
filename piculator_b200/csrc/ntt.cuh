// NTT engine: batched power-of-two number-theoretic transforms modulo
// 64-bit primes (< 2^63) on sm_100a.
//
// Forward = decimation in frequency, natural order in, bit-reversed order out.
// For primes c * 2^32 + 1 below 2^61 (lazy butterflies) forward outputs are
// only reduced to [0, 4p) and inverse outputs to [0, 8p); the consumers
// (Montgomery pointwise products of operands below 4p, the CRT's Shoup
// scaling of any 64-bit operand) accept them as they are.
// Inverse = decimation in time, bit-reversed in, natural out, unscaled.
// A convolution therefore never permutes: forward, pointwise, inverse.  The
// natural-order NTT of the reference (NNT::NTT, NTT.cpp:191-223) is forward +
// one bit-reversal permutation.
//
// Large lengths use the four-/six-step decomposition N = N1 * N2 (* N3):
// strided "column" passes (a size-N1 DIF over every column of an N1 x M tile,
// W columns per CTA so every global access is a W*8-byte run, then the
// inter-step twiddle w_(N1 M)^(col * k1)) and one contiguous "row" pass.  Each
// pass reads and writes the array once; inside a pass the butterflies run in
// radix-8 register groups with shared-memory exchanges between groups.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "modarith.cuh"

namespace pic {

constexpr int kInnerBits = 13;  // largest in-CTA sub-transform (2^13 points)
constexpr int kMaxPrimesPerBatch = 3;

// Device view of one prime's constants and twiddle tables.
struct PrimeDev {
    uint64_t p;
    uint64_t pinv_neg;
    uint64_t r2;
    int K;        // outer tables cover roots of order 2^K
    int S;        // outer split: e = hi * 2^S + lo
    int IB;       // inner table order bits (min(K, kInnerBits))
    int lazy;     // 1 when 8p < 2^64 and p = c 2^32 + 1: transforms keep values in [0, 4p) / [0, 8p)
    const uint64_t* inner_fwd;  // (w, w') Shoup pairs, w = root_(2^IB)^i, i < 2^(IB-1)
    const uint64_t* inner_inv;  // same for root^-1
    const uint64_t* olo_fwd;    // Montgomery form root_(2^K)^i, i < 2^S
    const uint64_t* ohi_fwd;    // Montgomery form root_(2^K)^(i 2^S), i < 2^(K-S)
    const uint64_t* olo_inv;
    const uint64_t* ohi_inv;
    // Lazy primes only (else null): the outer roots as Shoup pairs (w, w'),
    // same indexing as olo / ohi.
    const uint64_t* slo_fwd;
    const uint64_t* shi_fwd;
    const uint64_t* slo_inv;
    const uint64_t* shi_inv;
    // Lazy primes only (else null): inner roots by level, Shoup pairs.  The
    // roots of order 2^m (m = 1 .. 13), root^e for e < 2^(m-1), sit at pair
    // index 2^(m-1) - 1 + e, so consecutive e are consecutive pairs.
    const uint64_t* lvl_fwd;
    const uint64_t* lvl_inv;
    // floor(2^128 / p) = mu_hi 2^64 + mu_lo: Shoup companions on the device
    uint64_t mu_hi, mu_lo;
    // FP64 primes (below 2^47, the FP64 product form): residues are doubles
    // holding signed integers, and every table entry is the twiddle w as the
    // bits of one double (the level, outer and pass tables keep their indexing
    // with 8-byte entries).  Only the fast passes serve them.
    int fp64;
    double pd, pinv;  // p and fl(1 / p)
};

// Host-owned tables for one prime (built once, cached for the process).
struct PrimeTables {
    uint64_t p = 0, g = 0;
    int adicity = 0;
    PrimeDev dev{};
};

const PrimeTables& prime_tables(uint64_t p);

// The reference's prime for transform length 2^k (NTT.cpp:125-158).
uint64_t reference_prime(int k);
// The reference's generator rule: smallest primitive root (NTT.cpp:104-123).
uint64_t smallest_generator(uint64_t p);

// The three 62-bit primes of the multi-prime product (c * 2^32 + 1).
extern const uint64_t kProductPrimes[3];
// The three primes of the FP64 product form (c * 2^32 + 1 below 2^47).
extern const uint64_t kDblPrimes[3];
// Tables of an FP64 prime (p < 2^47, 2-adicity >= 13), cached like prime_tables.
const PrimeTables& dbl_prime_tables(uint64_t p);

// Product forms: the integer three-prime NTT (64-bit pieces, primes below
// 2^61, lazy Shoup butterflies) and the FP64 one (56-bit pieces, primes below
// 2^47, butterflies on the FP64 pipe).
enum NttForm { kFormInt = 0, kFormDbl = 1, kFormChosen = 2 };

// A batch of transforms of length 2^k laid out at data + i * stride
// (i < count); transform i uses prime[i / per_prime].
// A forward transform's input read straight from binary-splitting child
// slots instead of `data`: item i (prime i / per_prime, child
// c0 + i % per_prime) takes 64-bit pieces first + j of the child's words
// (cap words per slot, len[child] of them used, zero above), reduced mod the
// item's prime.  Only the first pass reads it; every pass writes `data`.
struct SplitSrc {
    const uint32_t* words = nullptr;  // null: the input is already in `data`
    const uint32_t* len = nullptr;
    uint32_t cap = 0;
    size_t c0 = 0;
    size_t first = 0;
};

struct NttBatch {
    uint64_t* data;
    size_t stride;
    int count;
    int per_prime;
    PrimeDev prime[kMaxPrimesPerBatch];
    SplitSrc src;
};

void ntt_forward_dif(const NttBatch& b, int k, cudaStream_t s);
void ntt_inverse_dit(const NttBatch& b, int k, cudaStream_t s);
void ntt_bitreverse(const NttBatch& b, int k, cudaStream_t s);

// out[i] = a[i] * b[i] * 2^-64 mod p over every transform of the batch
// (b may equal a for squaring); b's transforms are b_stride apart (0: a's
// stride).  FP64 primes: out[i] = a[i] * b[i] mod p (no Montgomery factor).
void ntt_pointwise_mont(const NttBatch& a, const uint64_t* b, int k, cudaStream_t s, size_t b_stride = 0);

// T[i] = T[i] * A[i] mod p exactly (reference ntt_pointwise semantics).
void ntt_pointwise_plain(uint64_t* T, const uint64_t* A, int k, const PrimeDev& P, cudaStream_t s);
// T[i] = T[i] * n^-1 mod p.
void ntt_scale_ninv(uint64_t* T, int k, const PrimeDev& P, cudaStream_t s);

// G lazy Shoup butterflies per second with operands in registers (ceiling.cu).
double butterfly_ceiling(cudaStream_t s);
// The same for the FP64 form's butterflies (about nine FP64 instructions each).
double butterfly_ceiling_dbl(cudaStream_t s);

// Pass split used for length 2^k (for reporting / tests).
std::vector<int> ntt_pass_bits(int k, int form = kFormInt);
// Tunable geometry per length and form (row-pass bits 8..13, column tile
// log2 width 0..6 with 0 = automatic, bits per register round 2..4; the FP64
// form runs only the fast passes: row bits 11..13, rounds of 3 or 4 bits).
void ntt_set_geometry(int k, int row_bits, int col_lw, int rbits, int form = kFormInt);
// FP64 column passes use per-point twiddle tables for blocks of at most
// 2^bits points (0: never), else the two-level tables.
void ntt_set_dbl_pass_bits(int bits);
int ntt_dbl_pass_bits();
// FP64 column passes of 2^5 .. 2^9 rows through the persistent kernel fed by
// TMA bulk copies, with tiles of at most 2^bits points (0: the
// one-tile-per-CTA kernel).
void ntt_set_cols_bulk(int bits);
int ntt_cols_bulk();
// True (and cleared) when a bulk-copy wait of a column pass timed out since
// the last call; synchronises with the device.
bool ntt_take_bulk_error();
void ntt_get_geometry(int k, int* row_bits, int* col_lw, int* rbits, int form = kFormInt);

}  // namespace pic
