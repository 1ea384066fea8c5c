// pic::BigFloat implementation (reference semantics, BigFloat.cpp:14-568).
#include <math.h>
#include <string.h>

#include <sstream>

#include "bigfloat.hpp"
#include "radix.cuh"
#include "linear.cuh"
#include "mul.cuh"

namespace pic {

static thread_local int t_mul_mode = PIC_MUL_AUTO;
void set_mul_mode(int mode) { t_mul_mode = mode; }
int get_mul_mode() { return t_mul_mode; }

static constexpr size_t kExtraPrecision = 2;  // YCL_BIGFLOAT_EXTRA_PRECISION, BigFloat.h:6

WordStore::~WordStore()
{
    if (base && initialized()) dev_free(base, bytes, ctx().stream);
}

std::shared_ptr<WordStore> alloc_words(size_t L)
{
    auto s = std::make_shared<WordStore>();
    s->bytes = (L ? L : 1) * sizeof(uint32_t);
    s->base = (uint32_t*)dev_alloc(s->bytes, ctx().stream);
    return s;
}

static cudaStream_t S() { return ctx().stream; }

// ---- construction / copies (BigFloat.cpp:14-79) ----------------------------
BigFloat::BigFloat() : sign(true), exp(0), L(0) {}

BigFloat::BigFloat(uint32_t x, bool sign_) : sign(true), exp(0), L(1)
{
    if (x == 0) {
        L = 0;
        return;
    }
    sign = sign_;
    store = alloc_words(1);
    PIC_CUDA(cudaMemcpyAsync(store->base, &x, sizeof(uint32_t), cudaMemcpyHostToDevice, S()));
    PIC_CUDA(cudaStreamSynchronize(S()));
    T = store->base;
}

BigFloat::BigFloat(BigFloat&& x) noexcept
    : sign(x.sign), exp(x.exp), L(x.L), T(x.T), store(std::move(x.store))
{
    x.sign = true;
    x.exp = 0;
    x.L = 0;
    x.T = nullptr;
}

BigFloat::BigFloat(const BigFloat& x) : sign(x.sign), exp(x.exp), L(x.L), T(x.T), store(x.store) {}

BigFloat& BigFloat::operator=(BigFloat&& x) noexcept
{
    sign = x.sign;
    exp = x.exp;
    L = x.L;
    T = x.T;
    store = std::move(x.store);
    x.sign = true;
    x.exp = 0;
    x.L = 0;
    x.T = nullptr;
    return *this;
}

BigFloat& BigFloat::operator=(const BigFloat& x)
{
    sign = x.sign;
    exp = x.exp;
    L = x.L;
    T = x.T;
    store = x.store;
    return *this;
}

BigFloat BigFloat::from_host(bool sign, int64_t exp, const uint32_t* words, size_t L)
{
    BigFloat z;
    z.sign = sign;
    z.exp = exp;
    z.L = L;
    if (L) {
        z.store = alloc_words(L);
        PIC_CUDA(cudaMemcpyAsync(z.store->base, words, L * sizeof(uint32_t), cudaMemcpyHostToDevice, S()));
        PIC_CUDA(cudaStreamSynchronize(S()));
        z.T = z.store->base;
    }
    return z;
}

BigFloat BigFloat::from_device(bool sign, int64_t exp, std::shared_ptr<WordStore> store, const uint32_t* ptr,
                               size_t L)
{
    BigFloat z;
    z.sign = sign;
    z.exp = exp;
    z.L = L;
    z.store = std::move(store);
    z.T = L ? ptr : nullptr;
    return z;
}

void BigFloat::to_host(uint32_t* words) const { read_words(words, T, L, S()); }

std::vector<uint32_t> BigFloat::words() const
{
    std::vector<uint32_t> w(L);
    to_host(w.data());
    return w;
}

// ---- getters (BigFloat.cpp:109-147) -------------------------------------------
uint32_t BigFloat::word_at(int64_t mag) const
{
    if (mag < exp) return 0;
    if (mag >= exp + (int64_t)L) return 0;
    uint32_t w;
    read_words(&w, T + (size_t)(mag - exp), 1, S());
    return w;
}

int BigFloat::ucmp(const BigFloat& x) const
{
    WordView a{T, exp, (int64_t)L}, b{x.T, x.exp, (int64_t)x.L};
    return lin_ucmp(a, b, S());
}

// ---- arithmetic ------------------------------------------------------------------
void BigFloat::negate()
{
    if (L == 0) return;
    sign = !sign;
}

// mul(uint32_t) -- BigFloat.cpp:156-183
BigFloat BigFloat::mul(uint32_t x) const
{
    if (L == 0 || x == 0) return BigFloat();
    auto st = alloc_words(L + 1);
    lin_mul_u32(st->base, T, L, x, S());
    uint32_t top;
    read_words(&top, st->base + L, 1, S());
    return from_device(sign, exp, st, st->base, top != 0 ? L + 1 : L);
}

// uadd -- BigFloat.cpp:184-232
BigFloat BigFloat::uadd(const BigFloat& x, size_t p) const
{
    const int64_t magA = exp + (int64_t)L, magB = x.exp + (int64_t)x.L;
    const int64_t top = magA > magB ? magA : magB;
    int64_t bot = exp < x.exp ? exp : x.exp;
    int64_t TL = top - bot;
    if (p == 0) p = (size_t)TL;
    else p += kExtraPrecision;
    if (TL > (int64_t)p) {
        bot = top - (int64_t)p;
        TL = (int64_t)p;
    }
    TL = (int64_t)(uint32_t)TL;  // the reference stores z.L = (uint32_t)TL
    auto st = alloc_words((size_t)TL + 1);
    WordView a{T, exp, (int64_t)L}, b{x.T, x.exp, (int64_t)x.L};
    lin_addsub(st->base, (size_t)TL, a, b, bot, false, st->base + TL, S());
    uint32_t carry;
    read_words(&carry, st->base + TL, 1, S());
    return from_device(sign, bot, st, st->base, (size_t)TL + (carry ? 1 : 0));
}

// usub -- BigFloat.cpp:233-287 (|this| >= |x|)
BigFloat BigFloat::usub(const BigFloat& x, size_t p) const
{
    const int64_t magA = exp + (int64_t)L, magB = x.exp + (int64_t)x.L;
    const int64_t top = magA > magB ? magA : magB;
    int64_t bot = exp < x.exp ? exp : x.exp;
    int64_t TL = top - bot;
    if (p == 0) p = (size_t)TL;
    else p += kExtraPrecision;
    if (TL > (int64_t)p) {
        bot = top - (int64_t)p;
        TL = (int64_t)p;
    }
    TL = (int64_t)(uint32_t)TL;
    auto st = alloc_words((size_t)TL + 1);
    WordView a{T, exp, (int64_t)L}, b{x.T, x.exp, (int64_t)x.L};
    lin_addsub(st->base, (size_t)TL, a, b, bot, true, st->base + TL, S());
    const size_t nz = lin_top_nonzero(st->base, (size_t)TL, S());
    if (nz == 0) return BigFloat();  // zero: exp 0, sign positive (BigFloat.cpp:280-284)
    return from_device(sign, bot, st, st->base, nz);
}

// add -- BigFloat.cpp:288-305
BigFloat BigFloat::add(const BigFloat& x, size_t p) const
{
    if (sign == x.sign) return uadd(x, p);
    if (ucmp(x) > 0) return usub(x, p);
    return x.usub(*this, p);
}

// sub -- BigFloat.cpp:306-325
BigFloat BigFloat::sub(const BigFloat& x, size_t p) const
{
    if (sign != x.sign) return uadd(x, p);
    if (ucmp(x) > 0) return usub(x, p);
    BigFloat z = x.usub(*this, p);
    z.negate();
    return z;
}

// mul -- BigFloat.cpp:326-444
BigFloat BigFloat::mul(const BigFloat& x, size_t p, int) const
{
    if (L == 0 || x.L == 0) return BigFloat();
    if (p == 0) p = L + x.L;
    else p += kExtraPrecision;
    int64_t Aexp = exp, Bexp = x.exp;
    size_t AL = L, BL = x.L;
    const uint32_t* AT = T;
    const uint32_t* BT = x.T;
    if (AL > p) {
        const size_t chop = AL - p;
        AL = p;
        Aexp += (int64_t)chop;
        AT += chop;
    }
    if (BL > p) {
        const size_t chop = BL - p;
        BL = p;
        Bexp += (int64_t)chop;
        BT += chop;
    }
    const size_t zl = AL + BL;
    auto st = alloc_words(zl);
    mul_dispatch(st->base, AT, AL, BT, BL, t_mul_mode, S());
    uint32_t top;
    read_words(&top, st->base + zl - 1, 1, S());
    return from_device(sign == x.sign, Aexp + Bexp, st, st->base, top == 0 ? zl - 1 : zl);
}

// rcp -- BigFloat.cpp:445-511
BigFloat BigFloat::rcp(size_t p, int threads) const
{
    if (L == 0) throw Error(PIC_ERR_DIVIDE_BY_ZERO, "Divide by Zero");
    if (p == 0) {
        int64_t Aexp = exp;
        size_t AL = L;
        const uint32_t* AT = T;
        if (AL > 3) {
            const size_t chop = AL - 3;
            AL = 3;
            Aexp += (int64_t)chop;
            AT += chop;
        }
        uint32_t w[3] = {0, 0, 0};
        read_words(w, AT, AL, S());
        // Host double seed, bit-identical to the reference's arithmetic.
        double val = (double)w[0];
        if (AL >= 2) val += (double)w[1] * 4294967296.;
        if (AL >= 3) val += (double)w[2] * 4294967296. * 4294967296.;
        val = 1. / val;
        Aexp = -Aexp;
        while (val < 4294967296.) {
            val *= 4294967296.;
            Aexp--;
        }
        const uint64_t v = (uint64_t)val;
        const uint32_t out[2] = {(uint32_t)v, (uint32_t)(v >> 32)};
        return from_host(sign, Aexp, out, 2);
    }
    size_t s = p / 2 + 1;
    if (p == 1) s = 0;
    if (p == 2) s = 1;
    BigFloat R = rcp(s, threads);
    // r1 = r0 - (r0 * x - 1) * r0 -- BigFloat.cpp:510.  Both products take
    // r0 whole (it is shorter than p + 2 words) at the same main transform
    // length, so its forward transform is made once.
    OperandHold hold(R.T, R.L);
    return R.sub(this->mul(R, p, threads).sub(BigFloat(1), p).mul(R, p, threads), p);
}

// div -- BigFloat.cpp:512-515
BigFloat BigFloat::div(const BigFloat& x, size_t p, int threads) const
{
    return this->mul(x.rcp(p, threads), p, threads);
}

// invsqrt -- BigFloat.cpp:516-568
BigFloat invsqrt(uint32_t x, size_t p, int threads)
{
    if (x == 0) throw Error(PIC_ERR_DIVIDE_BY_ZERO, "Divide by Zero");
    if (p == 0) {
        double val = 1. / sqrt((double)x);
        int64_t exponent = 0;
        while (val < 4294967296.) {
            val *= 4294967296.;
            exponent--;
        }
        const uint64_t v = (uint64_t)val;
        const uint32_t out[2] = {(uint32_t)v, (uint32_t)(v >> 32)};
        return BigFloat::from_host(true, exponent, out, 2);
    }
    size_t s = p / 2 + 1;
    if (p == 1) s = 0;
    if (p == 2) s = 1;
    BigFloat T = invsqrt(x, s, threads);
    OperandHold hold(T.T, T.L);                  // r0 is transformed once for r0^2 and (...) * r0
    BigFloat temp = T.mul(T, p, threads);        // r0^2
    // r0^2 * x: the reference forms it as temp.mul(BigFloat(x), 0), an exact
    // product with a one-word operand (BigFloat.cpp:562).  mul(uint32) gives
    // the same words, length, sign and exponent (BigFloat.cpp:156-183: exact
    // product, one carry word kept only when nonzero, as mul drops one zero
    // top word, :411-412) with one linear pass instead of three transforms.
    temp = temp.mul(x);
    temp = temp.sub(BigFloat(1), p);             // r0^2 * x - 1
    temp = temp.mul(2147483648u);                // (r0^2 * x - 1) / 2
    temp.exp--;
    temp = temp.mul(T, p, threads);              // (r0^2 * x - 1) / 2 * r0
    return T.sub(temp, p);                       // r0 - (r0^2 * x - 1) / 2 * r0
}

// ---- string conversion (BigFloat.cpp:83-106) -----------------------------------
__global__ void hex_words_kernel(char* out, const uint32_t* T, size_t top, size_t nw)
{
    // word loc = top - 1 - i  ->  out[8 i .. 8 i + 8) as %08x
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nw; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t w = T[top - 1 - i];
        char* o = out + 8 * i;
#pragma unroll
        for (int c = 0; c < 8; c++) {
            const uint32_t d = (w >> (28 - 4 * c)) & 15u;
            o[c] = (char)(d < 10 ? '0' + d : 'a' + d - 10);
        }
    }
}

size_t BigFloat::hex_into(size_t digits, char* out, size_t cap) const
{
    PIC_REQUIRE(L >= 1, PIC_ERR_INVALID, "to_string_hex of zero");
    const size_t nw = (digits + 7) / 8;
    PIC_REQUIRE(nw <= L - 1, PIC_ERR_INVALID, "to_string_hex: fewer words than digits requested");
    uint32_t topw;
    read_words(&topw, T + L - 1, 1, S());
    char prefix[16];
    const int np = snprintf(prefix, sizeof prefix, "%u.", topw);
    const size_t full = (size_t)np + 8 * nw;
    const size_t len = 2 + digits < full ? 2 + digits : full;
    PIC_REQUIRE(len + 1 <= cap, PIC_ERR_INVALID, "to_string_hex: output buffer too small");
    memcpy(out, prefix, (size_t)np < len ? (size_t)np : len);
    if (len > (size_t)np) {
        const size_t body = len - (size_t)np;  // hex characters to copy
        const size_t nwords = (body + 7) / 8;
        DevBuf<char> d(8 * nwords, S());
        hex_words_kernel<<<grid_for(nwords, 256), 256, 0, S()>>>(d.get(), T, L - 1, nwords);
        PIC_CHECK_LAUNCH();
        count_launch();
        PIC_CUDA(cudaMemcpyAsync(out + np, d.get(), body, cudaMemcpyDeviceToHost, S()));
        PIC_CUDA(cudaStreamSynchronize(S()));
    }
    out[len] = 0;
    return len;
}

std::string BigFloat::to_string_hex(size_t digits) const
{
    std::string s(2 + digits + 16, '\0');
    const size_t n = hex_into(digits, &s[0], s.size());
    s.resize(n);
    return s;
}

std::string BigFloat::to_string_dec(size_t digits) const
{
    // BigFloat.cpp:83-94 prints the fraction below the top word nine digits at
    // a time by clearing the top word and multiplying by 10^9 (O(n^2)); the
    // same digits come from one exact product and a divide-and-conquer split
    // by powers of 10^9 (radix.cu).
    return to_string_dec_fast(*this, digits);
}

}  // namespace pic
