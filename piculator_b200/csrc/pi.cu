// Pi() -- PI.h:138-212 -- on device-resident BigFloats.
//
// Two forms:
//  * plain  (PIC_PI_PLAIN): the reference's recursion node by node, every
//    product one three-prime NTT multiply (its own launch sequence, no
//    batching across products, no schoolbook);
//  * chosen (PIC_PI_CHOSEN): the lower binary-splitting levels evaluated level
//    by level in batched launches (bsr.cu), the upper levels and the Newton
//    phases through the tuned multiply.
// Both produce the reference's pi.txt byte for byte.
#include <math.h>
#include <string.h>

#include <chrono>

#include "bigfloat.hpp"
#include "bsr.cuh"
#include "checkpoint.cuh"
#include "common.cuh"
#include "mul.cuh"
#include "pi.cuh"
#include "ntt.cuh"

namespace pic {

// Sizes -- PI.h:141-144 (same double arithmetic).
void pi_sizes(uint64_t decimal_digits, uint64_t* hex_digits, uint64_t* p_words, uint64_t* terms)
{
    const size_t hex = (size_t)((double)decimal_digits * log(10) / log(16));
    const size_t p = (hex + 9) / 9;
    const size_t p_dec = (decimal_digits + 9) / 9;
    const size_t t = (size_t)((double)p_dec * 0.6346230241342037371474889163921741077188431452678) + 1;
    if (hex_digits) *hex_digits = hex;
    if (p_words) *p_words = p;
    if (terms) *terms = t;
}

// Pi_BSR -- PI.h:64-136, serial recursion (the reference's thread split does
// not change any result).
void bsr_recursive(BigFloat& P, BigFloat& Q, BigFloat& R, uint32_t a, uint32_t b, size_t p)
{
    if (b - a == 1) {
        // P = (13591409 + 545140134 b)(2b-1)(6b-5)(6b-1) (-1)^b -- PI.h:68-75
        P = BigFloat(b).mul(545140134u);
        P = P.add(BigFloat(13591409u));
        P = P.mul(2 * b - 1);
        P = P.mul(6 * b - 5);
        P = P.mul(6 * b - 1);
        if (b % 2 == 1) P.negate();
        // Q = 10939058860032000 b^3 -- PI.h:77-79
        Q = BigFloat(b);
        Q = Q.mul(b).mul(b).mul(26726400u).mul(409297880u);
        // R = (2b-1)(6b-5)(6b-1) -- PI.h:81-84
        R = BigFloat(2 * b - 1);
        R = R.mul(6 * b - 5);
        R = R.mul(6 * b - 1);
        return;
    }
    const uint32_t m = (a + b) / 2;
    BigFloat P0, Q0, R0, P1, Q1, R1;
    bsr_recursive(P0, Q0, R0, a, m, p);
    bsr_recursive(P1, Q1, R1, m, b, p);
    // PI.h:110-112
    P = P0.mul(Q1, p).add(P1.mul(R0, p), p);
    Q = Q0.mul(Q1, p);
    R = R0.mul(R1, p);
}

namespace {
struct PhaseTimer {
    cudaEvent_t e[8];
    int n = 0;
    PhaseTimer()
    {
        for (auto& x : e) PIC_CUDA(cudaEventCreate(&x));
    }
    ~PhaseTimer()
    {
        for (auto& x : e) cudaEventDestroy(x);
    }
    void mark()
    {
        PIC_CUDA(cudaEventRecord(e[n++], ctx().stream));
        timeline_mark("pi_phase", ctx().stream);
    }
    double secs(int i, int j)
    {
        float ms = 0;
        PIC_CUDA(cudaEventSynchronize(e[j]));
        PIC_CUDA(cudaEventElapsedTime(&ms, e[i], e[j]));
        return ms / 1000.0;
    }
};
}  // namespace

BigFloat pi_compute(uint64_t decimal_digits, int mode, pic_pi_stats* st)
{
    require_init();
    uint64_t hex, p, terms;
    pi_sizes(decimal_digits, &hex, &p, &terms);
    if ((uint32_t)terms != terms) throw Error(PIC_ERR_LIMIT, "Limit Exceeded");  // PI.h:150-151
    const uint64_t launches0 = ctx().launches.load();
    const uint64_t products0 = ctx().products.load();
    const uint64_t recompute0 = ctx().fft_recomputes.load();
    const uint64_t reuse0 = held_transform_reuses();
    fft_reset_max_err();
    const int saved_mode = get_mul_mode();
    set_mul_mode(mode == PIC_PI_PLAIN ? PIC_MUL_NTT3 : PIC_MUL_AUTO);
    // the chosen form peaks below 512 bytes per word of precision (merge
    // batches of at most 256, live nodes and the top levels' workspace);
    // hold that much in the pool before the first merge
    if (mode != PIC_PI_PLAIN) reserve_pool((size_t)p * 512, ctx().stream);
    PhaseTimer tm;
    BigFloat P, Q, R;
    try {
        // a resumed computation starts after the newest phase on disk; the
        // phases it skips are timed as zero
        const int done = checkpoint_resume(decimal_digits, p, &P, &Q);
        tm.mark();
        if (done < 1) {
            if (mode == PIC_PI_PLAIN) bsr_recursive(P, Q, R, 0, (uint32_t)terms, (size_t)p);
            else bsr_chosen(P, Q, R, 0, (uint32_t)terms, (size_t)p, /*need_root_R=*/false);
            if (tracing()) {
                PIC_CUDA(cudaStreamSynchronize(ctx().stream));
                fprintf(stderr, "{\"trace\": \"bsr_done\"}\n");
            }
            P = Q.mul(13591409u).add(P, (size_t)p);  // PI.h:180-181
            Q = Q.mul(4270934400u);
            checkpoint_save(1, decimal_digits, p, terms, &P, &Q);
        }
        tm.mark();
        if (done < 2) {
            P = Q.div(P, (size_t)p);                 // PI.h:189
            checkpoint_save(2, decimal_digits, p, terms, &P, nullptr);
        }
        tm.mark();
        if (done < 3) {
            Q = invsqrt(10005, (size_t)p);           // PI.h:194
            checkpoint_save(3, decimal_digits, p, terms, &P, &Q);
        }
        tm.mark();
        P = P.mul(Q, (size_t)p);                 // PI.h:199
        tm.mark();
    } catch (...) {
        set_mul_mode(saved_mode);
        throw;
    }
    set_mul_mode(saved_mode);
    timeline_dump();
    PIC_REQUIRE(!ntt_take_bulk_error(), PIC_ERR_TIMEOUT, "a bulk-copy wait of an NTT column pass timed out");
    if (st) {
        memset(st, 0, sizeof *st);
        st->hex_digits = hex;
        st->p_words = p;
        st->terms = terms;
        st->seconds_bsr = tm.secs(0, 1);
        st->seconds_div = tm.secs(1, 2);
        st->seconds_invsqrt = tm.secs(2, 3);
        st->seconds_final_mul = tm.secs(3, 4);
        st->seconds_total = tm.secs(0, 4);
        st->kernel_launches = ctx().launches.load() - launches0;
        st->products = ctx().products.load() - products0;
        st->fft_max_err = fft_max_err_seen();
        st->fft_recomputes = ctx().fft_recomputes.load() - recompute0;
        st->transform_reuses = held_transform_reuses() - reuse0;
    }
    return P;
}

}  // namespace pic
