/* pic_oracle.h -- CPU restatement of Piculator's multiply path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker that tests/, the smoke test
 * and bench.py's CPU-baseline leg compare the CUDA path against; nothing in the
 * product library links or calls it.  Every function restates one piece of the
 * reference (file:line in the .c file) in plain C.  The restatement itself is
 * pinned against the reference program compiled from its own sources
 * (oracle/_ref, see Makefile) and against golden vectors generated from it
 * (tests/golden/).
 */
#ifndef PIC_ORACLE_H
#define PIC_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same layout as the reference harness's RefBF: a BigFloat's fields
 * (BigFloat.h:33-36) with the words owned by the caller. */
typedef struct {
    int32_t sign;   /* 1 = positive or zero, 0 = negative */
    int64_t exp;    /* exponent in 32-bit words */
    uint64_t L;     /* number of words */
    uint32_t* T;    /* words, little-endian */
} OracleBF;

enum {
    ORACLE_MUL = 0, ORACLE_ADD = 1, ORACLE_SUB = 2, ORACLE_MUL_U32 = 3,
    ORACLE_RCP = 4, ORACLE_DIV = 5, ORACLE_INVSQRT = 6, ORACLE_UCMP = 7
};

/* How the exact product inside BigFloat::mul is formed.  Every mode yields
 * the same words (the product is exact); AUTO follows the reference's own
 * choice (FFT below k = 27, NTT from k = 27, BigFloat.cpp:380-441) with
 * schoolbook for short operands and an NTT recompute if the FFT's rounding
 * distance ever exceeds 0.25. */
enum { ORACLE_MODE_AUTO = 0, ORACLE_MODE_SCHOOL = 1, ORACLE_MODE_FFT = 2, ORACLE_MODE_NTT = 3 };

void oracle_set_mode(int mode);
int oracle_get_mode(void);

/* Mirrors ref_bf_op: returns 0, -1 (out capacity too small; out->L holds the
 * needed length), -2 (the reference would throw), or 10 + ucmp for ORACLE_UCMP. */
int oracle_bf_op(int op, const OracleBF* a, const OracleBF* b, uint64_t p,
                 uint64_t s, OracleBF* out, uint64_t cap);

/* Exact product z[0 .. na+nb) = a * b (no truncation, no length fix-up). */
void oracle_mul_words(const uint32_t* a, size_t na, const uint32_t* b, size_t nb,
                      uint32_t* z);

/* Natural-order NTT of length 2^k modulo the reference's prime for k, with the
 * reference's generator; inverse includes the 1/n scaling. */
int oracle_ntt(int k, int inverse, uint64_t* data, uint64_t* p_out,
               uint64_t* g_out, uint64_t* w_out);

/* The reference's FFT conventions over 2^k interleaved complex doubles:
 * op 0 = forward (exp(+i theta) twiddles, bit-reversed output),
 * op 1 = inverse (exp(-i theta), bit-reversed input, unscaled). */
int oracle_fft(int k, int op, double* data);

/* Max |x - round(x)| seen by the last FFT product, and how many FFT products
 * were recomputed by the NTT because that distance exceeded 0.25. */
double oracle_fft_last_max_err(void);
uint64_t oracle_fft_recomputes(void);

/* The reference's prime / generator for transform length 2^k (k = 11..42). */
uint64_t oracle_prime(int k);
uint64_t oracle_generator(uint64_t p);

/* Chudnovsky binary splitting over [a, b) at precision p (PI.h:64-136). */
int oracle_bsr(uint32_t a, uint32_t b, uint64_t p, OracleBF* P, OracleBF* Q,
               OracleBF* R, uint64_t cap);

/* Whole pi run (PI.h:138-212): writes the hex string the reference dumps
 * into pi.txt.  Returns its length, or -1 if cap is too small. */
int64_t oracle_pi_hex(uint64_t decimal_digits, char* buf, uint64_t cap);

/* Sizes used by Pi() (PI.h:141-144). */
void oracle_pi_sizes(uint64_t decimal_digits, uint64_t* hex_digits,
                     uint64_t* p_words, uint64_t* terms);

#ifdef __cplusplus
}
#endif
#endif
