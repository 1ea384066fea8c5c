// Decimal output: BigFloat::to_string_dec (BigFloat.cpp:83-94) in
// O(M(n) log n) on the GPU.
//
// The reference prints the top word in decimal, a '.', and then nine digits
// at a time: it clears the top word and multiplies by 10^9, n times over, an
// O(n^2) loop (never run on its pi path, which prints hex).  Clearing the top
// word and multiplying by 10^9 exactly means the groups it prints are the
// decimal expansion of the fraction F = M / 2^B held in the words below the
// top (M their integer, B = 32 (L - 1)), truncated after 9 G digits
// (G = ceil(digits / 9)).  Those digits are the D = 9 G digits of the integer
//     N = floor(M 10^D / 2^B) = floor(M 5^D / 2^(B - D)),
// zero-padded on the left.  Here:
//   1. 5^D by binary powering, one exact product M 5^D, one shift: N.
//   2. N is split top-down, level by level, into halves of whole groups:
//      N = q 10^(9h) + r with h groups in r, every item of a level divided by
//      the same T = 10^(9h) in one batch of products: q = floor(N V / 2^e)
//      with the scaled reciprocal V = floor(2^e / T) - 2, e = 2 bits(T) + 32
//      (from BigFloat::rcp), which is q or, when r < 2^-29 T, q - 1; r = N - q T;
//      items whose r reaches T (rare) take one exact correction.
//   3. Items of at most 64 groups (576 digits, 61 words) are converted by one
//      thread each with repeated division by 10^9, straight into the text.
// Levels are padded to 64 2^m groups; the padding is leading zero groups,
// which are not written.
#include <math.h>
#include <string.h>

#include <string>
#include <vector>

#include "bigfloat.hpp"
#include "carry.cuh"
#include "common.cuh"
#include "linear.cuh"
#include "mul.cuh"
#include "radix.cuh"

namespace pic {

constexpr uint32_t kTenNine = 1000000000u;
constexpr int kLeafGroups = 64;     // groups of nine digits per leaf item
constexpr int kLeafWords = 61;      // 10^576 < 2^1914 < 2^(32 * 60): 60 words + 1 spare
constexpr int kGuard = 32;          // guard bits of the scaled reciprocal
constexpr size_t kDecIPT = 8;       // words per thread in the batched borrow pass
constexpr size_t kDecThreads = 256;
constexpr size_t kDecWPC = kDecIPT * kDecThreads;

// Words that hold any number below 10^(9 g).
static size_t words_for_groups(size_t g)
{
    return (size_t)ceil((double)g * 9.0 * 3.3219280948873623 / 32.0) + 1;
}

// out item i word j = bits [32 j + off, 32 j + off + 32) of in item i (bits
// outside [0, 32 in_words) read as 0; off may be negative: a left shift).
__global__ void dec_shift_kernel(uint32_t* __restrict__ out, size_t out_stride, size_t out_words,
                                 const uint32_t* __restrict__ in, size_t in_stride, size_t in_words, size_t count,
                                 int64_t off)
{
    const size_t total = count * out_words;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < total; g += (size_t)gridDim.x * blockDim.x) {
        const size_t it = g / out_words, j = g - it * out_words;
        const uint32_t* x = in + it * in_stride;
        const int64_t b = (int64_t)(32 * j) + off;
        const int64_t w0 = b >= 0 ? b / 32 : -((-b + 31) / 32);
        const int r = (int)(b - 32 * w0);
        auto get = [&](int64_t w) -> uint32_t { return (w >= 0 && w < (int64_t)in_words) ? x[w] : 0u; };
        const uint32_t lo = get(w0);
        const uint32_t v = r ? ((lo >> r) | (get(w0 + 1) << (32 - r))) : lo;
        out[it * out_stride + j] = v;
    }
}

static void dec_shift(uint32_t* out, size_t out_stride, size_t out_words, const uint32_t* in, size_t in_stride,
                      size_t in_words, size_t count, int64_t off, cudaStream_t s)
{
    const size_t total = count * out_words;
    dec_shift_kernel<<<grid_for(total, 256), 256, 0, s>>>(out, out_stride, out_words, in, in_stride, in_words, count,
                                                          off);
    PIC_CHECK_LAUNCH();
    count_launch();
}

// r_i = (a_i - b_i) mod 2^(32 n) for `count` items, b shared when b_stride is 0.
// K1: raw differences, in-CTA borrows resolved, one (G, P) per CTA (G: borrow
// out of the CTA whatever comes in, P: a borrow in passes through).
__global__ void __launch_bounds__(kDecThreads) dec_sub_k1(uint32_t* __restrict__ r, size_t r_stride,
                                                          const uint32_t* __restrict__ a, size_t a_stride,
                                                          const uint32_t* __restrict__ b, size_t b_stride,
                                                          size_t b_words, size_t n, size_t cpi, uint32_t* agg)
{
    const size_t it = blockIdx.x / cpi, c = blockIdx.x - it * cpi;
    const size_t base = c * kDecWPC + threadIdx.x * kDecIPT;
    const uint32_t* x = a + it * a_stride;
    const uint32_t* y = b + it * b_stride;
    uint32_t d[kDecIPT], gg[kDecIPT];
    uint32_t acc = kGPIdentity;
#pragma unroll
    for (size_t u = 0; u < kDecIPT; u++) {
        const size_t i = base + u;
        const uint32_t xa = i < n ? x[i] : 0u, yb = (i < n && i < b_words) ? y[i] : 0u;
        d[u] = xa - yb;
        gg[u] = xa < yb;
        acc = gp_combine(acc, gg[u] | ((uint32_t)(d[u] == 0u) << 1));
    }
    uint32_t total;
    const uint32_t pre = block_gp_scan(acc, &total);
    uint32_t bin = pre & 1u;  // borrow into this thread's words from lower threads of the CTA
    uint32_t* z = r + it * r_stride;
#pragma unroll
    for (size_t u = 0; u < kDecIPT; u++) {
        const size_t i = base + u;
        if (i < n) z[i] = d[u] - bin;
        bin = gg[u] | ((uint32_t)(d[u] == 0u) & bin);
    }
    if (threadIdx.x == 0) agg[blockIdx.x] = total;
}

// K3: CTAs with a borrow in subtract it from their own words.
__global__ void dec_sub_ripple(uint32_t* r, size_t r_stride, size_t n, size_t cpi, const uint32_t* bin)
{
    if (bin[blockIdx.x] == 0) return;
    const size_t it = blockIdx.x / cpi, c = blockIdx.x - it * cpi;
    uint32_t* z = r + it * r_stride;
    const size_t b = c * kDecWPC, e = b + kDecWPC < n ? b + kDecWPC : n;
    unsigned long long mine = ~0ull;
    for (size_t i = b + threadIdx.x; i < e; i += blockDim.x)
        if (z[i] != 0u && i < mine) mine = i;
    const size_t f = (size_t)block_min_u64(mine);
    for (size_t i = b + threadIdx.x; i < e && i < f; i += blockDim.x) z[i] = 0xffffffffu;
    if (threadIdx.x == 0 && f < e) z[f] -= 1u;
}

static void dec_sub(uint32_t* r, size_t r_stride, const uint32_t* a, size_t a_stride, const uint32_t* b,
                    size_t b_stride, size_t b_words, size_t n, size_t count, cudaStream_t s)
{
    const size_t cpi = (n + kDecWPC - 1) / kDecWPC;
    DevBuf<uint32_t> agg(count * cpi, s);
    ProfScope ps(KC_LINEAR, 12.0 * (double)(count * n), s);
    dec_sub_k1<<<(unsigned)(count * cpi), kDecThreads, 0, s>>>(r, r_stride, a, a_stride, b, b_stride, b_words, n,
                                                              cpi, agg.get());
    PIC_CHECK_LAUNCH();
    carry_scan_segments(agg.get(), count, cpi, s);
    dec_sub_ripple<<<(unsigned)(count * cpi), 256, 0, s>>>(r, r_stride, n, cpi, agg.get());
    PIC_CHECK_LAUNCH();
    count_launch(2);
}

// hi[i] = 1 + the highest word index where item i of x differs from t (0:
// equal), over n words; t has t_words words (zero above).
__global__ void dec_diff_kernel(const uint32_t* __restrict__ x, size_t x_stride, const uint32_t* __restrict__ t,
                                size_t t_words, size_t n, size_t cpi, unsigned long long* hi)
{
    const size_t it = blockIdx.x / cpi, c = blockIdx.x - it * cpi;
    const uint32_t* y = x + it * x_stride;
    const size_t b = c * kDecWPC, e = b + kDecWPC < n ? b + kDecWPC : n;
    unsigned long long mine = 0;
    for (size_t i = b + threadIdx.x; i < e; i += blockDim.x) {
        const uint32_t tv = i < t_words ? t[i] : 0u;
        if (y[i] != tv) mine = i + 1;
    }
    mine = warp_max_u64(mine);
    if ((threadIdx.x & 31) == 0 && mine) atomicMax(hi + it, mine);
}

// ge[i] = item i >= t; *nge counts them.
__global__ void dec_ge_kernel(const uint32_t* __restrict__ x, size_t x_stride, const uint32_t* __restrict__ t,
                              size_t t_words, const unsigned long long* hi, size_t count, uint8_t* ge,
                              unsigned int* nge)
{
    for (size_t it = blockIdx.x * (size_t)blockDim.x + threadIdx.x; it < count; it += (size_t)gridDim.x * blockDim.x) {
        const unsigned long long h = hi[it];
        bool g = true;  // equal counts as >=
        if (h) {
            const size_t j = (size_t)h - 1;
            const uint32_t tv = j < t_words ? t[j] : 0u;
            g = x[it * x_stride + j] > tv;
        }
        ge[it] = g ? 1 : 0;
        if (g) atomicAdd(nge, 1u);
    }
}

// One thread per leaf item (< 10^(9 * 64), kLeafWords words): 64 groups by
// repeated division by 10^9, written as text.  Item i's groups are global
// groups i * 64 .. i * 64 + 63 (most significant first); the first `skip`
// global groups are leading padding and are not written.
__global__ void dec_leaf_kernel(const uint32_t* __restrict__ items, size_t stride, size_t count, size_t skip,
                                size_t out_groups, char* __restrict__ out)
{
    for (size_t it = blockIdx.x * (size_t)blockDim.x + threadIdx.x; it < count; it += (size_t)gridDim.x * blockDim.x) {
        uint32_t w[kLeafWords];
        const uint32_t* x = items + it * stride;
        int top = 0;
#pragma unroll
        for (int k = 0; k < kLeafWords; k++) {
            w[k] = x[k];
            if (w[k]) top = k + 1;
        }
        for (int gq = kLeafGroups - 1; gq >= 0; gq--) {
            // divide w[0 .. top) by 10^9; the remainder is the group at gq
            uint64_t rem = 0;
            for (int k = top - 1; k >= 0; k--) {
                const uint64_t cur = (rem << 32) | w[k];
                w[k] = (uint32_t)(cur / kTenNine);
                rem = cur % kTenNine;
            }
            while (top > 0 && w[top - 1] == 0) top--;
            const size_t G = it * kLeafGroups + (size_t)gq;
            if (G < skip || G - skip >= out_groups) continue;
            char* o = out + 9 * (G - skip);
            uint32_t v = (uint32_t)rem;
#pragma unroll
            for (int c = 8; c >= 0; c--) {
                o[c] = (char)('0' + v % 10u);
                v /= 10u;
            }
        }
    }
}

namespace {
// A natural number as device words (little-endian), owned.
struct Nat {
    std::shared_ptr<WordStore> st;
    size_t L = 0;
    uint32_t* w() const { return st ? st->base : nullptr; }
};

BigFloat as_bf(const Nat& n) { return BigFloat::from_device(true, 0, n.st, n.st->base, n.L); }

// 5^e by binary powering (exact products).
BigFloat pow5(uint64_t e)
{
    BigFloat r(5u);
    if (e == 0) return BigFloat(1u);
    int hb = 63;
    while (!((e >> hb) & 1)) hb--;
    for (int b = hb - 1; b >= 0; b--) {
        r = r.mul(r, 0);
        if ((e >> b) & 1) r = r.mul(5u);
    }
    return r;
}

// x 2^sh (sh >= 0 bits) as a plain word array of `words` words.
Nat shifted(const BigFloat& x, int64_t sh, size_t words, cudaStream_t s)
{
    Nat n;
    n.L = words;
    n.st = alloc_words(words);
    dec_shift(n.st->base, words, words, x.device_words(), 0, x.get_precision(), 1, -sh, s);
    return n;
}

size_t bit_length(const Nat& n, cudaStream_t s)
{
    const size_t top = lin_top_nonzero(n.w(), n.L, s);
    if (top == 0) return 0;
    uint32_t w;
    read_words(&w, n.w() + top - 1, 1, s);
    return 32 * (top - 1) + (32 - __builtin_clz(w));
}

struct Divisor {
    Nat T;        // 10^(9 h)
    size_t bits;  // bit length of T
    Nat V;        // floor(2^(2 bits + kGuard) / T) - 2
};

// The reciprocal of T = 10^(9 h): V from BigFloat::rcp at enough precision
// that its error is far below one unit of V, then two units off so that V
// never exceeds the true floor and the quotient estimate never exceeds the
// true quotient.
Divisor make_divisor(Nat T, cudaStream_t s)
{
    Divisor d;
    d.T = std::move(T);
    d.bits = bit_length(d.T, s);
    const size_t ebits = 2 * d.bits + kGuard;
    const size_t pw = (ebits + 31) / 32 + 4;
    const BigFloat R = as_bf(d.T).rcp(pw);
    const int64_t off = -(32 * R.get_exponent() + (int64_t)ebits);  // right shift of R's words
    const size_t vw = (d.bits + kGuard) / 32 + 3;
    Nat v;
    v.L = vw;
    v.st = alloc_words(vw);
    dec_shift(v.st->base, vw, vw, R.device_words(), 0, R.get_precision(), 1, off, s);
    d.V.L = vw;
    d.V.st = alloc_words(vw);
    const BigFloat two(2u);
    DevBuf<uint32_t> fin(1, s);
    lin_addsub(d.V.st->base, vw, WordView{v.st->base, 0, (int64_t)vw}, WordView{two.device_words(), 0, 1}, 0, true,
               fin.get(), s);
    return d;
}

// T_j = 10^(9 * 64 * 2^j) for j < m: T_0 = 5^576 2^576, then squares.
std::vector<Divisor> make_divisors(size_t m, cudaStream_t s)
{
    std::vector<Divisor> out;
    if (m == 0) return out;
    const uint64_t e0 = 9 * (uint64_t)kLeafGroups;
    Nat T = shifted(pow5(e0), (int64_t)e0, words_for_groups(kLeafGroups), s);
    for (size_t j = 0; j < m; j++) {
        Nat next;
        if (j + 1 < m) {
            const BigFloat sq = as_bf(T).mul(as_bf(T), 0);
            next = shifted(sq, 0, words_for_groups((size_t)kLeafGroups << (j + 1)), s);
        }
        out.push_back(make_divisor(std::move(T), s));
        T = std::move(next);
    }
    return out;
}

// z_i = a_i * b for `count` items (exact), z stride zs.
void products(uint32_t* z, size_t zs, const uint32_t* a, size_t as, size_t na, const uint32_t* b, size_t nb,
              size_t count, cudaStream_t s)
{
    if (count <= 16) {
        for (size_t i = 0; i < count; i++) mul_dispatch(z + i * zs, a + i * as, na, b, nb, PIC_MUL_AUTO, s);
        return;
    }
    std::vector<pic_mul_desc> d(count);
    for (size_t i = 0; i < count; i++) d[i] = pic_mul_desc{z + i * zs, a + i * as, b, na, nb};
    mul_batch(d.data(), count, PIC_MUL_AUTO, s);
}
}  // namespace

void dec_digits(const BigFloat& x, size_t groups, char* d_out)
{
    cudaStream_t s = ctx().stream;
    const size_t L = x.get_precision();
    if (groups == 0) return;
    size_t m = 0;
    while (((size_t)kLeafGroups << m) < groups) m++;
    const size_t Gp = (size_t)kLeafGroups << m;
    const uint64_t D = 9 * (uint64_t)groups;
    // N = floor(M 5^D / 2^(B - D)) with M the words below the top one
    const size_t capN = words_for_groups(Gp);
    DevBuf<uint32_t> cur(capN, s);
    if (L <= 1) {
        PIC_CUDA(cudaMemsetAsync(cur.get(), 0, 4 * capN, s));
    } else {
        const BigFloat M = BigFloat::from_device(true, 0, nullptr, x.device_words(), L - 1);
        const BigFloat X = M.mul(pow5(D), 0);
        const int64_t off = 32 * (int64_t)(L - 1) - (int64_t)D;
        dec_shift(cur.get(), capN, capN, X.device_words(), 0, X.get_precision(), 1, off, s);
    }
    // top-down splits: level l has 2^l items of 64 2^(m - l) groups, split by
    // T = 10^(9 * 64 * 2^(m - l - 1))
    const std::vector<Divisor> divs = make_divisors(m, s);
    size_t count = 1, cap = capN;
    for (size_t l = 0; l < m; l++) {
        const size_t hg = (size_t)kLeafGroups << (m - l - 1);  // groups in each half
        const Divisor& dv = divs[m - l - 1];
        const size_t ccap = words_for_groups(hg);
        const size_t tw = dv.T.L, vw = dv.V.L;
        DevBuf<uint32_t> nxt(2 * count * ccap, s);
        {
            // q_i = floor(N_i V / 2^(2 bits + guard)), into the even slots
            const size_t ys = cap + vw;
            DevBuf<uint32_t> Y(count * ys, s);
            products(Y.get(), ys, cur.get(), cap, cap, dv.V.w(), vw, count, s);
            dec_shift(nxt.get(), 2 * ccap, ccap, Y.get(), ys, ys, count, (int64_t)(2 * dv.bits + kGuard), s);
        }
        {
            // r_i = N_i - q_i T over the low ccap words (r < 2 T fits), odd slots
            const size_t zs = ccap + tw;
            DevBuf<uint32_t> Z(count * zs, s);
            products(Z.get(), zs, nxt.get(), 2 * ccap, ccap, dv.T.w(), tw, count, s);
            dec_sub(nxt.get() + ccap, 2 * ccap, cur.get(), cap, Z.get(), zs, zs, ccap, count, s);
        }
        {
            // the quotient estimate is q or q - 1: items with r >= T take one
            // more step (checked again; more than one step means a reciprocal
            // far off its bound, reported rather than looped on)
            const size_t cpi = (ccap + kDecWPC - 1) / kDecWPC;
            DevBuf<unsigned long long> hi(count, s);
            DevBuf<uint8_t> ge(count, s);
            DevBuf<unsigned int> nge(1, s);
            DevBuf<uint32_t> fin(1, s), d1(1, s);
            const uint32_t one = 1;
            PIC_CUDA(cudaMemcpyAsync(d1.get(), &one, 4, cudaMemcpyHostToDevice, s));
            for (int round = 0;; round++) {
                PIC_CUDA(cudaMemsetAsync(hi.get(), 0, 8 * count, s));
                PIC_CUDA(cudaMemsetAsync(nge.get(), 0, 4, s));
                dec_diff_kernel<<<(unsigned)(count * cpi), 256, 0, s>>>(nxt.get() + ccap, 2 * ccap, dv.T.w(), tw,
                                                                        ccap, cpi, hi.get());
                dec_ge_kernel<<<grid_for(count, 256), 256, 0, s>>>(nxt.get() + ccap, 2 * ccap, dv.T.w(), tw,
                                                                   hi.get(), count, ge.get(), nge.get());
                PIC_CHECK_LAUNCH();
                count_launch(2);
                uint32_t n_ge = 0;
                read_words(&n_ge, (const uint32_t*)nge.get(), 1, s);
                if (n_ge == 0) break;
                PIC_REQUIRE(round < 2, PIC_ERR_INVALID, "decimal split: quotient estimate off by more than one");
                std::vector<uint8_t> h(count);
                PIC_CUDA(cudaMemcpyAsync(h.data(), ge.get(), count, cudaMemcpyDeviceToHost, s));
                PIC_CUDA(cudaStreamSynchronize(s));
                for (size_t i = 0; i < count; i++) {
                    if (!h[i]) continue;
                    uint32_t* q = nxt.get() + 2 * i * ccap;
                    uint32_t* r = q + ccap;
                    lin_addsub(r, ccap, WordView{r, 0, (int64_t)ccap}, WordView{dv.T.w(), 0, (int64_t)tw}, 0, true,
                               fin.get(), s);
                    lin_addsub(q, ccap, WordView{q, 0, (int64_t)ccap}, WordView{d1.get(), 0, 1}, 0, false, fin.get(),
                               s);
                }
            }
        }
        cur = std::move(nxt);
        count *= 2;
        cap = ccap;
    }
    // leaves
    PIC_REQUIRE(cap <= (size_t)kLeafWords, PIC_ERR_INVALID, "decimal leaf wider than its kernel");
    DevBuf<uint32_t> leaf;
    const uint32_t* items = cur.get();
    if (cap < (size_t)kLeafWords) {  // widen to the kernel's fixed width
        leaf = DevBuf<uint32_t>(count * kLeafWords, s);
        dec_shift(leaf.get(), kLeafWords, kLeafWords, cur.get(), cap, cap, count, 0, s);
        items = leaf.get();
    }
    dec_leaf_kernel<<<grid_for(count, 128), 128, 0, s>>>(items, kLeafWords, count, Gp - groups, groups, d_out);
    PIC_CHECK_LAUNCH();
    count_launch();
}

std::string to_string_dec_fast(const BigFloat& x, size_t digits)
{
    const size_t L = x.get_precision();
    if (L == 0) throw Error(PIC_ERR_INVALID, "to_string_dec of an empty number");  // the reference reads T[L-1]
    uint32_t top = 0;
    read_words(&top, x.device_words() + L - 1, 1, ctx().stream);
    std::string s = std::to_string(top) + ".";
    const size_t groups = (digits + 8) / 9;
    if (groups) {
        DevBuf<char> d(9 * groups, ctx().stream);
        dec_digits(x, groups, d.get());
        std::string tail(9 * groups, '0');
        PIC_CUDA(cudaMemcpyAsync(&tail[0], d.get(), 9 * groups, cudaMemcpyDeviceToHost, ctx().stream));
        PIC_CUDA(cudaStreamSynchronize(ctx().stream));
        s += tail;
    }
    return s.substr(0, 2 + digits);
}

}  // namespace pic
