// extern "C" entry points of include/piculator_b200.h.  Each one converts
// internal exceptions into a pic_status and records the message for
// pic_last_error().
#include <string.h>

#include <memory>
#include <string>

#include "bigfloat.hpp"
#include "common.cuh"
#include "fft.cuh"
#include "mul.cuh"
#include "ntt.cuh"
#include "bsr.cuh"
#include "checkpoint.cuh"
#include "pi.cuh"
#include "transform.cuh"

namespace pic {
void profile_begin();
int profile_end(pic_kernel_stat* out, int cap);
void init_context(int device);
void shutdown_context();
void set_last_error(const std::string& s);
const std::string& last_error();
}  // namespace pic

using namespace pic;

struct pic_bigfloat_s {
    BigFloat v;
};

template <class F>
static pic_status guarded(F&& f)
{
    try {
        f();
        return PIC_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.status;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return PIC_ERR_NO_MEMORY;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return PIC_ERR_INVALID;
    }
}

static pic_bf wrap(BigFloat&& v)
{
    pic_bf h = new pic_bigfloat_s{std::move(v)};
    return h;
}

template <class F>
static void with_mode(int mode, F&& f)
{
    const int saved = get_mul_mode();
    set_mul_mode(mode);
    try {
        f();
    } catch (...) {
        set_mul_mode(saved);
        throw;
    }
    set_mul_mode(saved);
}

#define PIC_REQ_PTR(p) PIC_REQUIRE((p) != nullptr, PIC_ERR_INVALID, #p " is NULL")

extern "C" {

pic_status pic_init(int device)
{
    return guarded([&] { init_context(device); });
}

pic_status pic_shutdown(void)
{
    return guarded([&] { shutdown_context(); });
}

const char* pic_last_error(void) { return last_error().c_str(); }

const char* pic_status_string(pic_status s)
{
    switch (s) {
    case PIC_OK: return "ok";
    case PIC_ERR_INVALID: return "invalid argument";
    case PIC_ERR_LENGTH: return "FFT length is too small.";
    case PIC_ERR_DIVIDE_BY_ZERO: return "Divide by Zero";
    case PIC_ERR_LIMIT: return "Limit Exceeded";
    case PIC_ERR_CUDA: return "CUDA error";
    case PIC_ERR_NO_MEMORY: return "out of memory";
    case PIC_ERR_NOT_INITIALIZED: return "not initialised";
    case PIC_ERR_IO: return "Cannot Create File";
    case PIC_ERR_TIMEOUT: return "device wait timed out";
    case PIC_ERR_STOPPED: return "stopped after a checkpoint";
    }
    return "unknown status";
}

pic_status pic_synchronize(void)
{
    return guarded([&] {
        require_init();
        PIC_CUDA(cudaStreamSynchronize(ctx().stream));
        PIC_REQUIRE(!ntt_take_bulk_error(), PIC_ERR_TIMEOUT, "a bulk-copy wait of an NTT column pass timed out");
    });
}

uint64_t pic_device_bytes_in_use(void) { return ctx().bytes_in_use.load(); }

void pic_debug_fail_allocations(int n) { ctx().fail_allocs.store(n); }

uint64_t pic_debug_allocation_count(void) { return ctx().alloc_calls.load(); }

pic_stream pic_default_stream(void) { return initialized() ? (pic_stream)ctx().stream : nullptr; }

pic_status pic_profile_begin(void)
{
    return guarded([&] {
        require_init();
        profile_begin();
    });
}

pic_status pic_profile_end(pic_kernel_stat* out, int cap, int* n)
{
    return guarded([&] {
        require_init();
        const int m = profile_end(out, cap);
        if (n) *n = m;
    });
}

pic_status pic_measure_butterfly_rate(double* gbfly_per_s)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(gbfly_per_s);
        *gbfly_per_s = butterfly_ceiling(ctx().stream);
    });
}

pic_status pic_measure_butterfly_rate_form(int form, double* gbfly_per_s)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(gbfly_per_s);
        PIC_REQUIRE(form == 0 || form == 1, PIC_ERR_INVALID, "unknown product form");
        *gbfly_per_s = form == 1 ? butterfly_ceiling_dbl(ctx().stream) : butterfly_ceiling(ctx().stream);
    });
}

// ---- NTT.h ---------------------------------------------------------------------
static PrimeDev ref_prime_dev(int k)
{
    PIC_REQUIRE(k >= 1 && k <= 32, PIC_ERR_INVALID, "k out of range (1..32)");
    return prime_tables(reference_prime(k)).dev;
}

static NttBatch single(uint64_t* T, int k, const PrimeDev& P)
{
    NttBatch b;
    b.data = T;
    b.stride = (size_t)1 << k;
    b.count = 1;
    b.per_prime = 1;
    b.prime[0] = P;
    return b;
}

pic_status pic_ntt_ensure_table(int k)
{
    return guarded([&] {
        require_init();
        ref_prime_dev(k);
    });
}

pic_status pic_ntt_forward(uint64_t* T, int k, pic_stream s)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(T);
        const PrimeDev P = ref_prime_dev(k);
        NttBatch b = single(T, k, P);
        ntt_forward_dif(b, k, resolve(s));
        ntt_bitreverse(b, k, resolve(s));
    });
}

pic_status pic_ntt_inverse(uint64_t* T, int k, pic_stream s)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(T);
        const PrimeDev P = ref_prime_dev(k);
        NttBatch b = single(T, k, P);
        ntt_bitreverse(b, k, resolve(s));
        ntt_inverse_dit(b, k, resolve(s));
        ntt_scale_ninv(T, k, P, resolve(s));  // rN, NTT.cpp:83
    });
}

pic_status pic_ntt_pointwise(uint64_t* T, const uint64_t* A, int k, pic_stream s)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(T);
        PIC_REQ_PTR(A);
        ntt_pointwise_plain(T, A, k, ref_prime_dev(k), resolve(s));
    });
}

pic_status pic_int_to_ntt(uint64_t* T, int k, const uint32_t* A, size_t AL, pic_stream s)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(T);
        PIC_REQUIRE(AL == 0 || A, PIC_ERR_INVALID, "A is NULL");
        PIC_REQUIRE(k >= 1 && k <= 32, PIC_ERR_INVALID, "k out of range");
        int_to_ntt_dev(T, k, A, AL, resolve(s));
    });
}

pic_status pic_ntt_to_int(const uint64_t* T, int k, uint32_t* A, size_t AL, pic_stream s)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(T);
        PIC_REQUIRE(AL == 0 || A, PIC_ERR_INVALID, "A is NULL");
        PIC_REQUIRE(k >= 1 && k <= 32, PIC_ERR_INVALID, "k out of range");
        ntt_to_int_dev(T, k, A, AL, resolve(s));
    });
}

uint64_t pic_ntt_prime(int k) { return (k >= 1 && k <= 42) ? reference_prime(k) : 0; }

// ---- FFT.h ---------------------------------------------------------------------
pic_status pic_fft_ensure_table(int k)
{
    return guarded([&] {
        require_init();
        PIC_REQUIRE(k >= 1 && k <= 30, PIC_ERR_INVALID, "k out of range (1..30)");
    });
}

pic_status pic_fft_forward(double* T, int k, pic_stream s)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(T);
        fft_forward_dif(FftBatch{(double2*)T, (size_t)1 << k, 1}, k, resolve(s));
    });
}

pic_status pic_fft_inverse(double* T, int k, pic_stream s)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(T);
        fft_inverse_dit(FftBatch{(double2*)T, (size_t)1 << k, 1}, k, resolve(s));
    });
}

pic_status pic_fft_pointwise(double* T, const double* A, int k, pic_stream s)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(T);
        PIC_REQ_PTR(A);
        PIC_REQUIRE(k >= 1 && k <= 30, PIC_ERR_INVALID, "k out of range (1..30)");
        fft_pointwise((double2*)T, (const double2*)A, (size_t)1 << k, resolve(s));
    });
}

pic_status pic_int_to_fft(double* T, int k, const uint32_t* A, size_t AL, pic_stream s)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(T);
        PIC_REQUIRE(k >= 1 && k <= 30, PIC_ERR_INVALID, "k out of range (1..30)");
        PIC_REQUIRE(((size_t)1 << k) >= 4 * AL, PIC_ERR_LENGTH, "FFT length is too small.");  // FFT.cpp:500-501
        fft_split((double2*)T, k, A, AL, 8, resolve(s));
    });
}

pic_status pic_fft_to_int(const double* T, int k, uint32_t* A, size_t AL, pic_stream s)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(T);
        PIC_REQUIRE(k >= 1 && k <= 30, PIC_ERR_INVALID, "k out of range (1..30)");
        PIC_REQUIRE(((size_t)1 << k) >= 4 * AL, PIC_ERR_LENGTH, "FFT length is too small.");  // FFT.cpp:535-536
        const double e = fft_coef_to_words((const double2*)T, 4 * AL, 1.0 / (double)((size_t)1 << k), 8, A, AL,
                                           resolve(s));
        fft_note_max_err(e);
    });
}

double pic_fft_last_max_err(void) { return fft_last_max_err(); }

int pic_fft_piece_bits(int k) { return k < 1 || k > 62 ? 0 : fft_piece_bits(k); }

double pic_fft_error_bound(int k, int bits)
{
    return k < 1 || k > 62 || bits < 1 || bits > 32 ? -1.0 : fft_error_bound(k, bits);
}

uint64_t pic_fft_recompute_count(void) { return ctx().fft_recomputes.load(); }

uint64_t pic_product_count(void) { return ctx().products.load(); }

// ---- products -----------------------------------------------------------------
pic_status pic_mul(uint32_t* z, const uint32_t* a, size_t na, const uint32_t* b, size_t nb, int mode,
                   pic_stream s)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(z);
        PIC_REQ_PTR(a);
        PIC_REQ_PTR(b);
        PIC_REQUIRE(na > 0 && nb > 0, PIC_ERR_INVALID, "empty operand");
        mul_dispatch(z, a, na, b, nb, mode, resolve(s));
    });
}

pic_status pic_mul_batch(const pic_mul_desc* d, size_t count, int mode, pic_stream s)
{
    return guarded([&] {
        require_init();
        PIC_REQUIRE(count == 0 || d, PIC_ERR_INVALID, "descs is NULL");
        mul_batch(d, count, mode, resolve(s));
    });
}

pic_status pic_mul_noalloc(uint32_t* z, const uint32_t* a, size_t na, const uint32_t* b, size_t nb, pic_stream s)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(z);
        PIC_REQ_PTR(a);
        PIC_REQ_PTR(b);
        PIC_REQUIRE(na > 0 && nb > 0, PIC_ERR_INVALID, "empty operand");
        mul_noalloc(z, a, na, b, nb, resolve(s));
    });
}

pic_status pic_mul_host(uint32_t* z, const uint32_t* a, size_t na, const uint32_t* b, size_t nb, int mode)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(z);
        PIC_REQ_PTR(a);
        PIC_REQ_PTR(b);
        PIC_REQUIRE(na > 0 && nb > 0, PIC_ERR_INVALID, "empty operand");
        cudaStream_t st = ctx().stream;
        DevBuf<uint32_t> da(na, st), db(nb, st), dz(na + nb, st);
        PIC_CUDA(cudaMemcpyAsync(da.get(), a, na * 4, cudaMemcpyHostToDevice, st));
        PIC_CUDA(cudaMemcpyAsync(db.get(), b, nb * 4, cudaMemcpyHostToDevice, st));
        mul_dispatch(dz.get(), da.get(), na, db.get(), nb, mode, st);
        PIC_CUDA(cudaMemcpyAsync(z, dz.get(), (na + nb) * 4, cudaMemcpyDeviceToHost, st));
        PIC_CUDA(cudaStreamSynchronize(st));
    });
}

// ---- BigFloat handles ------------------------------------------------------------
pic_status pic_bf_from_words(pic_bf* out, int sign, int64_t exp, const uint32_t* words, size_t L)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(out);
        PIC_REQUIRE(L == 0 || words, PIC_ERR_INVALID, "words is NULL");
        *out = wrap(BigFloat::from_host(sign != 0, exp, words, L));
    });
}

pic_status pic_bf_from_u32(pic_bf* out, uint32_t x, int sign)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(out);
        *out = wrap(BigFloat(x, sign != 0));
    });
}

pic_status pic_bf_free(pic_bf x)
{
    return guarded([&] { delete x; });
}

pic_status pic_bf_info(pic_bf x, int* sign, int64_t* exp, size_t* L)
{
    return guarded([&] {
        PIC_REQ_PTR(x);
        if (sign) *sign = x->v.get_sign() ? 1 : 0;
        if (exp) *exp = x->v.get_exponent();
        if (L) *L = x->v.get_precision();
    });
}

pic_status pic_bf_to_words(pic_bf x, uint32_t* words, size_t cap)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(x);
        PIC_REQUIRE(cap >= x->v.get_precision(), PIC_ERR_INVALID, "capacity too small");
        if (x->v.get_precision()) x->v.to_host(words);
    });
}

// Orders `to` after all work queued so far on `from` (no host wait).
static void stream_after(cudaStream_t to, cudaStream_t from)
{
    if (to == from) return;
    cudaEvent_t e;
    PIC_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    PIC_CUDA(cudaEventRecord(e, from));
    PIC_CUDA(cudaStreamWaitEvent(to, e, 0));
    PIC_CUDA(cudaEventDestroy(e));
}

pic_status pic_bf_to_device(pic_bf x, uint32_t* dst, size_t cap, pic_stream s)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(x);
        const size_t L = x->v.get_precision();
        PIC_REQUIRE(cap >= L, PIC_ERR_INVALID, "capacity too small");
        PIC_REQUIRE(L == 0 || dst, PIC_ERR_INVALID, "dst is NULL");
        if (!L) return;
        const cudaStream_t cs = resolve(s);
        stream_after(cs, ctx().stream);  // the words are written on the library's stream
        PIC_CUDA(cudaMemcpyAsync(dst, x->v.device_words(), L * sizeof(uint32_t), cudaMemcpyDeviceToDevice, cs));
        stream_after(ctx().stream, cs);  // later library work may not free the words before the copy
    });
}

pic_status pic_bf_from_device(pic_bf* out, int sign, int64_t exp, const uint32_t* src, size_t L, pic_stream s)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(out);
        PIC_REQUIRE(L == 0 || src, PIC_ERR_INVALID, "src is NULL");
        if (L == 0) {
            *out = wrap(BigFloat());
            return;
        }
        auto st = alloc_words(L);
        stream_after(ctx().stream, resolve(s));  // src is complete on the caller's stream
        PIC_CUDA(cudaMemcpyAsync(st->base, src, L * sizeof(uint32_t), cudaMemcpyDeviceToDevice, ctx().stream));
        stream_after(resolve(s), ctx().stream);  // the caller may reuse src after this point on s
        *out = wrap(BigFloat::from_device(sign != 0, exp, st, st->base, L));
    });
}

pic_status pic_bf_to_dec(pic_bf x, size_t digits, char* buf, size_t cap)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(x);
        PIC_REQ_PTR(buf);
        const std::string s = x->v.to_string_dec(digits);
        PIC_REQUIRE(s.size() + 1 <= cap, PIC_ERR_INVALID, "buffer too small");
        memcpy(buf, s.c_str(), s.size() + 1);
    });
}

pic_status pic_bf_negate(pic_bf x)
{
    return guarded([&] {
        PIC_REQ_PTR(x);
        x->v.negate();
    });
}

pic_status pic_bf_mul_u32(pic_bf* out, pic_bf a, uint32_t x)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(out);
        PIC_REQ_PTR(a);
        *out = wrap(a->v.mul(x));
    });
}

pic_status pic_bf_add(pic_bf* out, pic_bf a, pic_bf b, size_t p)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(out);
        PIC_REQ_PTR(a);
        PIC_REQ_PTR(b);
        *out = wrap(a->v.add(b->v, p));
    });
}

pic_status pic_bf_sub(pic_bf* out, pic_bf a, pic_bf b, size_t p)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(out);
        PIC_REQ_PTR(a);
        PIC_REQ_PTR(b);
        *out = wrap(a->v.sub(b->v, p));
    });
}

pic_status pic_bf_mul(pic_bf* out, pic_bf a, pic_bf b, size_t p, int mode)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(out);
        PIC_REQ_PTR(a);
        PIC_REQ_PTR(b);
        with_mode(mode, [&] { *out = wrap(a->v.mul(b->v, p)); });
    });
}

pic_status pic_bf_rcp(pic_bf* out, pic_bf a, size_t p, int mode)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(out);
        PIC_REQ_PTR(a);
        with_mode(mode, [&] { *out = wrap(a->v.rcp(p)); });
    });
}

pic_status pic_bf_div(pic_bf* out, pic_bf a, pic_bf b, size_t p, int mode)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(out);
        PIC_REQ_PTR(a);
        PIC_REQ_PTR(b);
        with_mode(mode, [&] { *out = wrap(a->v.div(b->v, p)); });
    });
}

pic_status pic_bf_invsqrt(pic_bf* out, uint32_t x, size_t p, int mode)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(out);
        with_mode(mode, [&] { *out = wrap(invsqrt(x, p)); });
    });
}

int pic_bf_ucmp(pic_bf a, pic_bf b)
{
    int r = 0;
    pic_status st = guarded([&] {
        require_init();
        PIC_REQ_PTR(a);
        PIC_REQ_PTR(b);
        r = a->v.ucmp(b->v);
    });
    return st == PIC_OK ? r : -2;
}

pic_status pic_bf_to_hex(pic_bf x, size_t digits, char* buf, size_t cap)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(x);
        PIC_REQ_PTR(buf);
        x->v.hex_into(digits, buf, cap);
    });
}

// ---- Transform.h ----------------------------------------------------------------
struct pic_transform_s {
    TransformOperand t;
};

pic_status pic_transform_create(pic_transform* out, pic_bf x, size_t p, int k)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(out);
        PIC_REQ_PTR(x);
        *out = new pic_transform_s{transform_create(x->v, p, k)};
    });
}

pic_status pic_transform_mul(pic_transform t1, pic_transform t2)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(t1);
        PIC_REQ_PTR(t2);
        transform_mul(t1->t, t2->t);
    });
}

pic_status pic_transform_to_bf(pic_bf* out, pic_transform t)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(out);
        PIC_REQ_PTR(t);
        *out = wrap(transform_to_bigfloat(t->t));
    });
}

pic_status pic_transform_free(pic_transform t)
{
    return guarded([&] { delete t; });
}

// ---- Pi -------------------------------------------------------------------------
pic_status pic_bsr(uint32_t a, uint32_t b, size_t p, int mode, pic_bf* P, pic_bf* Q, pic_bf* R)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(P);
        PIC_REQ_PTR(Q);
        PIC_REQ_PTR(R);
        PIC_REQUIRE(b > a, PIC_ERR_INVALID, "empty range");
        PIC_REQUIRE(mode == PIC_PI_CHOSEN || mode == PIC_PI_PLAIN, PIC_ERR_INVALID, "unknown mode");
        BigFloat p_, q_, r_;
        with_mode(mode == PIC_PI_PLAIN ? PIC_MUL_NTT3 : PIC_MUL_AUTO, [&] {
            if (mode == PIC_PI_PLAIN) bsr_recursive(p_, q_, r_, a, b, p);
            else bsr_chosen(p_, q_, r_, a, b, p);
        });
        *P = wrap(std::move(p_));
        *Q = wrap(std::move(q_));
        *R = wrap(std::move(r_));
    });
}

pic_status pic_set_tuning(int knob, int64_t value)
{
    return guarded([&] {
        PIC_REQUIRE(value >= 0, PIC_ERR_INVALID, "tuning value must be >= 0");
        switch (knob) {
        case PIC_TUNE_BSR_SCHOOL_MAX: bsr_set_school_threshold((uint32_t)value); break;
        case PIC_TUNE_MUL_SCHOOL_MAX: mul_set_thresholds(value, -1); break;
        case PIC_TUNE_MUL_FFT_MAX: mul_set_thresholds(-1, value); break;
        case PIC_TUNE_BATCH_GRAPHS: mul_batch_set_graphs(value != 0); break;
        case PIC_TUNE_BSR_WRAP: bsr_set_wrap(value != 0); break;
        case PIC_TUNE_MUL_WRAP: mul_set_wrap(value != 0); break;
        case PIC_TUNE_BSR_COMBINE: bsr_set_combine(value != 0); break;
        case PIC_TUNE_BSR_SMALL_MERGE:
            PIC_REQUIRE(value <= 2, PIC_ERR_INVALID, "small-merge mode is 0, 1 or 2");
            bsr_set_small_merge((int)value);
            break;
        case PIC_TUNE_BSR_KARATSUBA:
            PIC_REQUIRE(value == 0 || (value >= 4 && value <= 4096), PIC_ERR_INVALID,
                        "Karatsuba threshold is 0 or 4..4096 words");
            bsr_set_karatsuba((uint32_t)value);
            break;
        case PIC_TUNE_FFT_ACCEPT_PPM:
            PIC_REQUIRE(value <= 500000, PIC_ERR_INVALID, "FFT acceptance is at most 500000 ppm (0.5)");
            mul_set_fft_accept((double)value * 1e-6);
            break;
        case PIC_TUNE_NTT_FORM:
            PIC_REQUIRE(value <= 2, PIC_ERR_INVALID, "product form is 0 (integer), 1 (FP64) or 2 (chosen per product)");
            mul_set_ntt_form((int)value);
            break;
        case PIC_TUNE_COLS_BULK:
            PIC_REQUIRE(value == 0 || (value >= 8 && value <= 12), PIC_ERR_INVALID,
                        "bulk column tiles are 2^8 .. 2^12 points (0: off)");
            ntt_set_cols_bulk((int)value);
            break;
        case PIC_TUNE_DBL_PASS_TABLES:
            PIC_REQUIRE(value <= 24, PIC_ERR_INVALID, "FP64 pass-table bits are 0..24");
            ntt_set_dbl_pass_bits((int)value);
            break;
        default: throw Error(PIC_ERR_INVALID, "unknown tuning knob");
        }
    });
}

pic_status pic_set_ntt_geometry(int k, int row_bits, int col_width_log2, int radix_log2)
{
    return guarded([&] { ntt_set_geometry(k, row_bits, col_width_log2, radix_log2); });
}

pic_status pic_get_ntt_geometry(int k, int* row_bits, int* col_width_log2, int* radix_log2)
{
    return guarded([&] {
        PIC_REQ_PTR(row_bits);
        PIC_REQ_PTR(col_width_log2);
        PIC_REQ_PTR(radix_log2);
        ntt_get_geometry(k, row_bits, col_width_log2, radix_log2);
    });
}

pic_status pic_set_ntt_geometry_form(int form, int k, int row_bits, int col_width_log2, int radix_log2)
{
    return guarded([&] { ntt_set_geometry(k, row_bits, col_width_log2, radix_log2, form); });
}

pic_status pic_get_ntt_geometry_form(int form, int k, int* row_bits, int* col_width_log2, int* radix_log2)
{
    return guarded([&] {
        PIC_REQ_PTR(row_bits);
        PIC_REQ_PTR(col_width_log2);
        PIC_REQ_PTR(radix_log2);
        PIC_REQUIRE(form == 0 || form == 1, PIC_ERR_INVALID, "unknown product form");
        ntt_get_geometry(k, row_bits, col_width_log2, radix_log2, form);
    });
}

int64_t pic_get_tuning(int knob)
{
    switch (knob) {
    case PIC_TUNE_BSR_SCHOOL_MAX: return bsr_school_threshold();
    case PIC_TUNE_MUL_SCHOOL_MAX: return mul_school_max();
    case PIC_TUNE_MUL_FFT_MAX: return mul_fft_max();
    case PIC_TUNE_BATCH_GRAPHS: return 1;
    case PIC_TUNE_BSR_WRAP: return bsr_wrap() ? 1 : 0;
    case PIC_TUNE_BSR_SMALL_MERGE: return bsr_small_merge();
    case PIC_TUNE_MUL_WRAP: return mul_wrap() ? 1 : 0;
    case PIC_TUNE_BSR_COMBINE: return bsr_combine() ? 1 : 0;
    case PIC_TUNE_FFT_ACCEPT_PPM: return (int64_t)llround(mul_fft_accept() * 1e6);
    case PIC_TUNE_BSR_KARATSUBA: return bsr_karatsuba();
    case PIC_TUNE_NTT_FORM: return mul_ntt_form();
    case PIC_TUNE_DBL_PASS_TABLES: return ntt_dbl_pass_bits();
    case PIC_TUNE_COLS_BULK: return ntt_cols_bulk();
    }
    return -1;
}

pic_status pic_pi_sizes(uint64_t d, uint64_t* hex_digits, uint64_t* p_words, uint64_t* terms)
{
    return guarded([&] { pi_sizes(d, hex_digits, p_words, terms); });
}

pic_status pic_pi_compute(uint64_t decimal_digits, int mode, pic_bf* out, pic_pi_stats* stats)
{
    return guarded([&] {
        require_init();
        PIC_REQ_PTR(out);
        PIC_REQUIRE(mode == PIC_PI_CHOSEN || mode == PIC_PI_PLAIN, PIC_ERR_INVALID, "unknown pi mode");
        pic_pi_stats local;
        BigFloat P = pi_compute(decimal_digits, mode, &local);
        *out = wrap(std::move(P));
        if (stats) *stats = local;
    });
}

pic_status pic_pi_set_checkpoint(const char* dir, int flags)
{
    return guarded([&] {
        PIC_REQUIRE((flags & ~(PIC_CKPT_WRITE | PIC_CKPT_RESUME)) == 0, PIC_ERR_INVALID, "unknown checkpoint flags");
        checkpoint_configure(dir, flags);
    });
}

pic_status pic_checkpoint_inspect(const char* path, uint64_t* digits, uint64_t* p_words, uint32_t* phase, int verify)
{
    return guarded([&] {
        PIC_REQ_PTR(path);
        if (checkpoint_inspect_file(path, digits, p_words, phase, verify != 0, nullptr) != 0)
            throw Error(PIC_ERR_IO, std::string("checkpoint ") + path + ": cannot open");
    });
}

void pic_debug_stop_after_phase(int phase) { checkpoint_debug_stop_after(phase); }

pic_status pic_pi_hex(uint64_t decimal_digits, int mode, char* out, size_t cap, size_t* out_len,
                      pic_pi_stats* stats)
{
    return guarded([&] {
        require_init();
        PIC_REQUIRE(mode == PIC_PI_CHOSEN || mode == PIC_PI_PLAIN, PIC_ERR_INVALID, "unknown pi mode");
        pic_pi_stats local;
        BigFloat P = pi_compute(decimal_digits, mode, &local);
        uint64_t hex;
        pi_sizes(decimal_digits, &hex, nullptr, nullptr);
        if (out) {
            cudaEvent_t e0, e1;
            PIC_CUDA(cudaEventCreate(&e0));
            PIC_CUDA(cudaEventCreate(&e1));
            PIC_CUDA(cudaEventRecord(e0, ctx().stream));
            const size_t n = P.hex_into((size_t)hex, out, cap);  // to_string_hex, PI.h:204
            PIC_CUDA(cudaEventRecord(e1, ctx().stream));
            PIC_CUDA(cudaEventSynchronize(e1));
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            local.seconds_hex = ms / 1000.0;
            if (out_len) *out_len = n;
        }
        if (stats) *stats = local;
    });
}

}  // extern "C"
