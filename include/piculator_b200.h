/* piculator_b200.h -- C ABI of the B200 multiply engine for Piculator.
 *
 * Plain pointers and sizes only.  Every entry point returns a pic_status (the
 * reference throws string literals instead; the mapping is listed on
 * pic_status).  Device pointers are CUDA global-memory pointers on the device
 * given to pic_init; host pointers are ordinary host memory.  Calls that take
 * a pic_stream are ordered on that stream (NULL = the library's own stream);
 * everything else is synchronous.  The library is thread-safe after pic_init
 * (one internal lock serialises host-side bookkeeping).
 *
 * Reference interfaces replaced (file:line in vayun-mathur/Piculator):
 *   NTT.h:4-9        ntt_* C API                   -> pic_ntt_*
 *   FFT.h:4-9        fft_* C API                   -> pic_fft_*
 *   Transform.h:5-33 Transform / mulNTT / mulFFT   -> pic_transform_*
 *   BigFloat.h:8-46  class BigFloat (+ invsqrt)    -> pic_bf_* (handles)
 *   BigFloat.cpp:326-444 BigFloat::mul's product   -> pic_mul, pic_mul_batch
 *   PI.h:138-212     Pi(digits, threads)           -> pic_pi_hex
 */
#ifndef PICULATOR_B200_H
#define PICULATOR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PIC_OK = 0,
    PIC_ERR_INVALID = 1,         /* bad argument (null pointer, k out of range, ...) */
    PIC_ERR_LENGTH = 2,          /* "FFT length is too small." FFT.cpp:501,536 NTT.cpp:353 */
    PIC_ERR_DIVIDE_BY_ZERO = 3,  /* "Divide by Zero" BigFloat.cpp:451,524 */
    PIC_ERR_LIMIT = 4,           /* "Limit Exceeded" PI.h:150-151 */
    PIC_ERR_CUDA = 5,            /* a CUDA runtime call failed (see pic_last_error) */
    PIC_ERR_NO_MEMORY = 6,       /* device or pinned-host allocation failed */
    PIC_ERR_NOT_INITIALIZED = 7, /* pic_init has not succeeded */
    PIC_ERR_IO = 8,              /* "Cannot Create File" PI.h:42 */
    PIC_ERR_TIMEOUT = 9,         /* a bounded device-side wait gave up */
    PIC_ERR_STOPPED = 10         /* stopped by pic_debug_stop_after_phase (checkpoint tests) */
} pic_status;

typedef void* pic_stream; /* a cudaStream_t */

/* ---- library ------------------------------------------------------------ */
pic_status pic_init(int device);
pic_status pic_shutdown(void);
const char* pic_last_error(void);
const char* pic_status_string(pic_status s);
pic_status pic_synchronize(void);
/* Device bytes currently held by the library's pool and by live handles. */
uint64_t pic_device_bytes_in_use(void);

/* The library's own stream (a cudaStream_t), for callers that time or order
 * work against it. */
pic_stream pic_default_stream(void);

/* Live kernel timing: between begin and end every instrumented launch is
 * bracketed by CUDA events on its stream; end reports, per kernel class, the
 * launches, summed device seconds and summed algorithmic bytes.  *n receives
 * the number of classes (entries beyond cap are dropped). */
typedef struct {
    char name[24];
    uint64_t launches;
    double seconds;
    double bytes;
} pic_kernel_stat;
pic_status pic_profile_begin(void);
pic_status pic_profile_end(pic_kernel_stat* out, int cap, int* n);

/* The integer roofline of the NTT passes on this GPU: lazy 64-bit Shoup
 * butterflies per second (in G) with operands in registers and no memory
 * traffic.  No reference counterpart (a measurement aid). */
pic_status pic_measure_butterfly_rate(double* gbfly_per_s);
/* The same per product form: 0 the integer butterflies above, 1 the FP64
 * form's (FP64 modular products, about nine FP64 instructions each). */
pic_status pic_measure_butterfly_rate_form(int form, double* gbfly_per_s);

/* Test hook: make the next n device allocations fail with PIC_ERR_NO_MEMORY
 * (host-side fault injection; no GPU fault is involved). */
void pic_debug_fail_allocations(int n);
/* Test hook: how many allocations the library has made so far -- pool
 * allocations, direct cudaMalloc of twiddle tables, pinned host staging.
 * No reference counterpart (lets tests prove a path allocates nothing). */
uint64_t pic_debug_allocation_count(void);

/* ---- NTT.h:4-9 -- natural-order NTT mod the reference's prime for k ------ */
/* T, A: device arrays of 2^k uint64 residues.  Same results word for word
 * as the reference's ntt_forward / ntt_inverse / ntt_pointwise (prime table
 * NTT.cpp:125-158, smallest generator NTT.cpp:104-123), for 11 <= k <= 32
 * (the reference itself only serves k >= 27, NTT.cpp:299). */
pic_status pic_ntt_ensure_table(int k);                                /* NTT.h:4 */
pic_status pic_ntt_forward(uint64_t* T, int k, pic_stream s);          /* NTT.h:5 */
pic_status pic_ntt_inverse(uint64_t* T, int k, pic_stream s);          /* NTT.h:6 */
pic_status pic_ntt_pointwise(uint64_t* T, const uint64_t* A, int k,
                             pic_stream s);                            /* NTT.h:7 */
pic_status pic_int_to_ntt(uint64_t* T, int k, const uint32_t* A, size_t AL,
                          pic_stream s);                               /* NTT.h:8 */
pic_status pic_ntt_to_int(const uint64_t* T, int k, uint32_t* A, size_t AL,
                          pic_stream s);                               /* NTT.h:9 */
uint64_t pic_ntt_prime(int k); /* the reference's prime for 2^k (NTT.cpp:178) */

/* ---- FFT.h:4-9 -- complex FP64 FFT, the reference's conventions ---------- */
/* T, A: device arrays of 2^k complex doubles, interleaved (re, im).  forward
 * is DIF with exp(+i theta) twiddles and bit-reversed output (FFT.cpp:64);
 * inverse is DIT, bit-reversed in, natural out, unscaled (FFT.cpp:266).
 * pic_fft_to_int rounds half up after scaling by 2^-k (FFT.cpp:520-571) and
 * records the largest |x - round(x)| it saw (pic_fft_last_max_err). */
pic_status pic_fft_ensure_table(int k);                                /* FFT.h:4 */
pic_status pic_fft_forward(double* T, int k, pic_stream s);            /* FFT.h:5 */
pic_status pic_fft_inverse(double* T, int k, pic_stream s);            /* FFT.h:6 */
pic_status pic_fft_pointwise(double* T, const double* A, int k,
                             pic_stream s);                            /* FFT.h:7 */
pic_status pic_int_to_fft(double* T, int k, const uint32_t* A, size_t AL,
                          pic_stream s);                               /* FFT.h:8 */
pic_status pic_fft_to_int(const double* T, int k, uint32_t* A, size_t AL,
                          pic_stream s);                               /* FFT.h:9 */
double pic_fft_last_max_err(void);
/* The piece width FFT products use at transform length 2^k (one real piece
 * per complex point): the widest b in 8..16 whose worst-case rounding error,
 * pic_fft_error_bound(k, b), stays below 1/4; 0 when none does (k >= 27).
 * Host arithmetic only, callable before pic_init.  No reference counterpart:
 * the reference always packs 8-bit pieces and never bounds the error
 * (FFT.cpp:485-519). */
int pic_fft_piece_bits(int k);
/* Worst-case rounding error of a length-2^k FFT convolution of b-bit pieces
 * (C. Percival, Math. Comp. 72 (2003), Theorem 5.1, with twiddle error
 * 2.5 * 2^-53); -1 for k outside 1..62 or bits outside 1..32. */
double pic_fft_error_bound(int k, int bits);
/* FFT products whose largest rounding distance passed the acceptance
 * threshold (0.25 unless PIC_TUNE_FFT_ACCEPT_PPM lowers it) and were
 * recomputed with the exact three-prime NTT, since pic_init.  No reference
 * counterpart: the reference never checks its FFT's rounding (FFT.cpp:520-571). */
uint64_t pic_fft_recompute_count(void);
/* Multi-word products formed since pic_init, whatever the kernel (pic_mul
 * calls, batched products, four per binary-splitting merge). */
uint64_t pic_product_count(void);

/* ---- whole products (the core of BigFloat::mul, BigFloat.cpp:413-487) ---- */
/* z[0 .. na+nb) = a * b exactly, device words, little-endian base 2^32.
 * z must not overlap a or b.  Any mode gives identical words. */
enum {
    PIC_MUL_AUTO = 0,     /* per-size choice from the tuned size classes */
    PIC_MUL_NTT_REF = 1,  /* the reference's layout: 16-bit points, one prime,
                             length 2^k >= 4(na+nb) (BigFloat.cpp:380-385) */
    PIC_MUL_NTT3 = 2,     /* three 62-bit primes, 64-bit points, CRT */
    PIC_MUL_FFT = 3,      /* FP64 FFT, limb split from the rounding bound,
                             NTT recompute when max distance > 0.25 */
    PIC_MUL_SCHOOL = 4,   /* batched schoolbook (short operands) */
    PIC_MUL_NTT3D = 5     /* three primes below 2^47, 56-bit points, FP64 butterflies, CRT */
};
pic_status pic_mul(uint32_t* z, const uint32_t* a, size_t na, const uint32_t* b,
                   size_t nb, int mode, pic_stream s);

/* Many independent products in one call (device pointers in each record).
 * The descriptor array itself is host memory.  Short products run in one
 * persistent schoolbook launch, the rest in batched three-prime NTT size
 * classes; the launch sequence is captured as a CUDA graph and replayed when
 * a later call has the same sizes.  Returns after the products are written. */
typedef struct {
    uint32_t* z;
    const uint32_t* a;
    const uint32_t* b;
    uint64_t na;
    uint64_t nb;
} pic_mul_desc;
pic_status pic_mul_batch(const pic_mul_desc* descs, size_t count, int mode,
                         pic_stream s);

/* Allocation-free product.  No counterpart in the reference: this exists for
 * callers that cannot allocate device memory when they multiply (an
 * application that has given its device memory to its own pool, a
 * latency-critical loop that must not take the allocator's locks or risk an
 * out-of-memory failure mid-computation).  Same result as pic_mul, computed
 * with the three-prime NTT in fixed storage compiled into the library
 * (about 3.5 MiB per GPU, held until the process exits).  Limit:
 * ceil(na/2) + ceil(nb/2) - 1 <= 65536 (about 131,000 product words);
 * longer products return PIC_ERR_LENGTH.  Calls share that storage, so calls
 * that overlap on the GPU race.  The first call on each device sets up the
 * storage (resolving its device address, filling twiddle tables) and
 * synchronises the stream: make that first call outside any stream capture. */
pic_status pic_mul_noalloc(uint32_t* z, const uint32_t* a, size_t na,
                           const uint32_t* b, size_t nb, pic_stream s);

/* Host-buffer convenience: copies in, multiplies, copies out (synchronous). */
pic_status pic_mul_host(uint32_t* z, const uint32_t* a, size_t na,
                        const uint32_t* b, size_t nb, int mode);

/* ---- BigFloat (BigFloat.h:8-46) as device-resident handles -------------- */
/* Semantics are the reference's exactly: sign/exp/L/T with exp counted in
 * 32-bit words, precision p in words with 2 guard words
 * (YCL_BIGFLOAT_EXTRA_PRECISION, BigFloat.h:6), p == 0 meaning exact. */
typedef struct pic_bigfloat_s* pic_bf;

pic_status pic_bf_from_words(pic_bf* out, int sign, int64_t exp,
                             const uint32_t* words_host, size_t L);
pic_status pic_bf_from_u32(pic_bf* out, uint32_t x, int sign); /* BigFloat.cpp:64 */
pic_status pic_bf_free(pic_bf x);
pic_status pic_bf_info(pic_bf x, int* sign, int64_t* exp, size_t* L);
pic_status pic_bf_to_words(pic_bf x, uint32_t* words_host, size_t cap);
/* Device-to-device word copies, for callers that move numbers between GPUs
 * themselves (the multi-GPU binary splitting sends them over NCCL).  dst and
 * src are device pointers on the library's device; the copies are ordered on
 * s after the library's pending work.  No reference counterpart. */
pic_status pic_bf_to_device(pic_bf x, uint32_t* dst, size_t cap, pic_stream s);
pic_status pic_bf_from_device(pic_bf* out, int sign, int64_t exp, const uint32_t* src,
                              size_t L, pic_stream s);
pic_status pic_bf_negate(pic_bf x);                                  /* :150 */
pic_status pic_bf_mul_u32(pic_bf* out, pic_bf a, uint32_t x);        /* :156 */
pic_status pic_bf_add(pic_bf* out, pic_bf a, pic_bf b, size_t p);    /* :288 */
pic_status pic_bf_sub(pic_bf* out, pic_bf a, pic_bf b, size_t p);    /* :306 */
pic_status pic_bf_mul(pic_bf* out, pic_bf a, pic_bf b, size_t p, int mode); /* :326 */
pic_status pic_bf_rcp(pic_bf* out, pic_bf a, size_t p, int mode);    /* :445 */
pic_status pic_bf_div(pic_bf* out, pic_bf a, pic_bf b, size_t p, int mode); /* :512 */
pic_status pic_bf_invsqrt(pic_bf* out, uint32_t x, size_t p, int mode); /* :516 */
int pic_bf_ucmp(pic_bf a, pic_bf b);                                  /* :123 */
pic_status pic_bf_to_hex(pic_bf x, size_t digits, char* buf, size_t cap); /* :95 */
/* to_string_dec (BigFloat.cpp:83): the top word in decimal, '.', then the
 * first `digits` decimal digits of the fraction below it -- the reference's
 * text exactly, computed in O(M(n) log n) instead of its O(n^2) loop. */
pic_status pic_bf_to_dec(pic_bf x, size_t digits, char* buf, size_t cap); /* :83 */

/* ---- Transform.h:5-33 -- transform-domain operands ----------------------- */
/* A pic_transform holds one operand's forward transform (three-prime form)
 * plus the BigFloat metadata of Transform.h:5-11, so a factor used in several
 * products is transformed once.  mul accumulates pointwise like mulNTT. */
typedef struct pic_transform_s* pic_transform;
pic_status pic_transform_create(pic_transform* out, pic_bf x, size_t p, int k);
pic_status pic_transform_mul(pic_transform t1, pic_transform t2); /* mulNTT, Transform.h:13-18 */
pic_status pic_transform_to_bf(pic_bf* out, pic_transform t);
pic_status pic_transform_free(pic_transform t);                    /* deleteNTT, :27-29 */

/* ---- Pi (PI.h:138-212) ---------------------------------------------------- */
enum {
    PIC_PI_CHOSEN = 0, /* batched binary-splitting levels + tuned products */
    PIC_PI_PLAIN = 1   /* one BigFloat::mul per product, each its own three-prime
                          NTT launch sequence (no batching, no schoolbook) */
};
typedef struct {
    uint64_t hex_digits;   /* PI.h:141 */
    uint64_t p_words;      /* PI.h:142 */
    uint64_t terms;        /* PI.h:144 */
    double seconds_bsr;    /* device time per phase (CUDA events) */
    double seconds_div;
    double seconds_invsqrt;
    double seconds_final_mul;
    double seconds_hex;
    double seconds_total;
    uint64_t kernel_launches;
    uint64_t products;     /* products formed: four per merge above the binary splitting's
                              bottom depth, plus every BigFloat product (the bottom depth's
                              merges of two leaves, done in registers, are not counted) */
    double fft_max_err;    /* largest FFT rounding distance seen */
    uint64_t fft_recomputes;
    uint64_t transform_reuses; /* Newton products that reused the iterate's forward transform */
} pic_pi_stats;

/* Computes pi to decimal_digits and writes the text the reference dumps into
 * pi.txt (to_string_hex, PI.h:204) into out (host), NUL-terminated.  Set
 * out = NULL to compute without copying the digits back. */
pic_status pic_pi_hex(uint64_t decimal_digits, int mode, char* out, size_t cap,
                      size_t* out_len, pic_pi_stats* stats);

/* Pi() without the final text: the result stays on the device as a BigFloat
 * handle (free it with pic_bf_free; pic_bf_to_hex gives the text). */
pic_status pic_pi_compute(uint64_t decimal_digits, int mode, pic_bf* out,
                          pic_pi_stats* stats);

/* Checkpoint / resume.  No reference counterpart: the reference keeps its
 * state in RAM only (PI.h:165-166) and a failed run starts over.  With a
 * directory set, pic_pi_hex / pic_pi_compute write <dir>/pi_<digits>.ckpt at
 * the end of each phase of Pi() -- 1: binary splitting and the combination
 * of PI.h:179-181 (P, Q), 2: the division of PI.h:189 (P), 3: the inverse
 * square root of PI.h:194 (P, Q) -- replacing the previous file only once the
 * new one is complete; with PIC_CKPT_RESUME a computation of the same digit
 * count starts after the newest phase found there.  A file that fails its
 * checks is reported (PIC_ERR_IO), never used.  dir = NULL turns it off. */
enum { PIC_CKPT_WRITE = 1, PIC_CKPT_RESUME = 2 };
pic_status pic_pi_set_checkpoint(const char* dir, int flags);
/* Reads a checkpoint file on the host (no GPU needed): its digit count,
 * working precision and phase; verify != 0 also checks every stored number
 * against its hash.  PIC_ERR_IO if it is not a valid checkpoint. */
pic_status pic_checkpoint_inspect(const char* path, uint64_t* digits, uint64_t* p_words,
                                  uint32_t* phase, int verify);
/* Test hook: after writing the checkpoint of `phase` (1..3), the computation
 * stops with PIC_ERR_STOPPED, as a crash right after it would (0 = never). */
void pic_debug_stop_after_phase(int phase);

/* Binary splitting over [a, b) at precision p (Pi_BSR, PI.h:64-136): the
 * batched form (PIC_PI_CHOSEN) or the node-by-node recursion (PIC_PI_PLAIN).
 * Both give the reference's P, Q, R word for word. */
pic_status pic_bsr(uint32_t a, uint32_t b, size_t p, int mode, pic_bf* P, pic_bf* Q,
                   pic_bf* R);

/* Tuning knobs (the size-class thresholds the autotuner sets). */
enum {
    PIC_TUNE_BSR_SCHOOL_MAX = 0, /* children up to this many words: CTA schoolbook merge */
    PIC_TUNE_MUL_SCHOOL_MAX = 1, /* products up to this many words: schoolbook in AUTO */
    PIC_TUNE_MUL_FFT_MAX = 2,    /* products up to this many words: FP64 FFT in AUTO (0: never) */
    PIC_TUNE_BATCH_GRAPHS = 3,   /* 1: pic_mul_batch replays captured CUDA graphs (default) */
    PIC_TUNE_BSR_WRAP = 4,       /* 1: binary-splitting NTT merges use wrapped products (default) */
    PIC_TUNE_BSR_SMALL_MERGE = 5, /* short schoolbook levels: 0 CTA, 1 + warp, 2 + thread per parent (default) */
    PIC_TUNE_MUL_WRAP = 6,        /* 1: three-prime products use the wrapped form when it is shorter (default) */
    PIC_TUNE_BSR_COMBINE = 7,     /* 1: binary-splitting NTT merges form P in the transform domain (default) */
    PIC_TUNE_FFT_ACCEPT_PPM = 8,  /* FFT products whose max rounding distance exceeds value * 1e-6 are
                                     recomputed with NTT3 (default 250000 = 0.25; lower it to test the
                                     recompute path) */
    PIC_TUNE_BSR_KARATSUBA = 9,   /* CTA schoolbook merges take one Karatsuba level for operands of at
                                     least this many words (0 = never) */
    PIC_TUNE_NTT_FORM = 10,       /* three-prime form of AUTO products and binary-splitting merges:
                                     0 integer (PIC_MUL_NTT3), 1 FP64 (PIC_MUL_NTT3D), 2 chosen per
                                     product (or merge level) by the transform work of the two forms */
    PIC_TUNE_DBL_PASS_TABLES = 11, /* FP64 column passes over blocks of at most 2^value points (0..24,
                                     default 20) stream per-point twiddle tables; longer blocks form the
                                     twiddles from the two-level tables */
    PIC_TUNE_COLS_BULK = 12       /* 8..12: FP64 column passes of 2^5 .. 2^9 rows run the persistent
                                     kernel whose tiles (at most 2^value points) arrive by TMA bulk
                                     copies (bounded waits: a wait past ~1 s of SM clocks ends the pass
                                     with PIC_ERR_TIMEOUT); 0 (default): one tile per CTA */
};
pic_status pic_set_tuning(int knob, int64_t value);
int64_t pic_get_tuning(int knob);

/* NTT geometry for transforms of length 2^k: bits handled by the contiguous
 * row pass (8..13), log2 columns per CTA in column passes (2..6, 0 = automatic)
 * and bits per register round (2..4, i.e. radix 4, 8 or 16). */
pic_status pic_set_ntt_geometry(int k, int row_bits, int col_width_log2, int radix_log2);
pic_status pic_get_ntt_geometry(int k, int* row_bits, int* col_width_log2, int* radix_log2);
/* The same per product form (0 integer, 1 FP64; the FP64 form takes row bits
 * 11..13 and radix bits 3..4, its passes having no general fallback). */
pic_status pic_set_ntt_geometry_form(int form, int k, int row_bits, int col_width_log2, int radix_log2);
pic_status pic_get_ntt_geometry_form(int form, int k, int* row_bits, int* col_width_log2, int* radix_log2);

/* Sizes Pi() derives from the digit count (PI.h:141-144). */
pic_status pic_pi_sizes(uint64_t decimal_digits, uint64_t* hex_digits,
                        uint64_t* p_words, uint64_t* terms);

#ifdef __cplusplus
}
#endif
#endif /* PICULATOR_B200_H */
