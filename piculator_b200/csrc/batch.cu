// Batched uneven products (pic_mul_batch): many independent products of
// different lengths in one call -- the shape of the lower binary-splitting
// levels (PI.h:110-112 over thousands of nodes), exposed for any caller.
//
// Plan per call:
//   * products of at most kSchoolMaxWords words go to one persistent
//     schoolbook launch: a grid of at most 148 x 8 CTAs pulls product indices
//     from an atomic counter (longest first) until the list is exhausted;
//   * the rest are binned by transform length 2^k (three-prime NTT, 64-bit
//     pieces); each bin is one batched split, forward, pointwise, inverse and
//     CRT sequence for all its products, then a scatter to their outputs.
// The launch sequence of a plan is captured once into a CUDA graph and
// replayed for later calls with the same sizes: only the descriptor table
// (device pointers and lengths) is re-uploaded before the replay.
#include <string.h>

#include <algorithm>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "carry.cuh"
#include "common.cuh"
#include "mul.cuh"
#include "ntt.cuh"

namespace pic {

struct DevDesc {
    uint32_t* z;
    const uint32_t* a;
    const uint32_t* b;
    uint32_t na, nb;
};

// ---- persistent schoolbook ------------------------------------------------------
constexpr int kPSchThreads = 256;

__global__ void __launch_bounds__(kPSchThreads) school_persistent_kernel(const DevDesc* __restrict__ d,
                                                                         const uint32_t* __restrict__ order,
                                                                         uint32_t n, uint32_t* counter)
{
    extern __shared__ uint32_t sm[];
    __shared__ uint32_t s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1u);
        __syncthreads();
        const uint32_t it = s_item;
        __syncthreads();
        if (it >= n) return;
        const DevDesc D = d[order[it]];
        const uint32_t na = D.na, nb = D.nb, zw = na + nb;
        uint32_t* sa = sm;
        uint32_t* sb = sa + na;
        uint32_t* col = sb + nb;
        for (uint32_t i = threadIdx.x; i < na; i += blockDim.x) sa[i] = D.a[i];
        for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) sb[i] = D.b[i];
        __syncthreads();
        for (uint32_t c = threadIdx.x; c < zw; c += blockDim.x) {
            uint64_t lo = 0;
            uint32_t hi = 0;
            if (c + 1 < zw) {
                const uint32_t i_lo = c + 1 > nb ? c + 1 - nb : 0;
                const uint32_t i_hi = c < na - 1 ? c : na - 1;
                for (uint32_t i = i_lo; i <= i_hi; i++) {
                    const uint64_t pr = (uint64_t)sa[i] * sb[c - i];
                    lo += pr;
                    hi += (lo < pr);
                }
            }
            col[3 * c] = (uint32_t)lo;
            col[3 * c + 1] = (uint32_t)(lo >> 32);
            col[3 * c + 2] = hi;
        }
        __syncthreads();
        const uint32_t per = (zw + blockDim.x - 1) / blockDim.x;
        const uint32_t w0 = threadIdx.x * per, w1 = min(w0 + per, zw);
        auto digit = [&](uint32_t w, uint32_t& g) -> uint32_t {
            uint64_t sw = col[3 * w], sp = 0;
            if (w >= 1) {
                sw += col[3 * (w - 1) + 1];
                sp += col[3 * (w - 1)];
            }
            if (w >= 2) {
                sw += col[3 * (w - 2) + 2];
                sp += col[3 * (w - 2) + 1];
            }
            if (w >= 3) sp += col[3 * (w - 3) + 2];
            const uint64_t t = (sw & 0xffffffffu) + (sp >> 32);
            g = (uint32_t)(t >> 32);
            return (uint32_t)t;
        };
        uint32_t gp = kGPIdentity;
        for (uint32_t w = w0; w < w1; w++) {
            uint32_t g;
            const uint32_t dd = digit(w, g);
            gp = gp_combine(gp, g | ((uint32_t)(dd == 0xffffffffu) << 1));
        }
        uint32_t total;
        uint32_t cin = block_gp_scan(gp, &total) & 1u;
        for (uint32_t w = w0; w < w1; w++) {
            uint32_t g;
            const uint32_t dd = digit(w, g);
            D.z[w] = dd + cin;
            cin = g | ((uint32_t)(dd == 0xffffffffu) & cin);
        }
        __syncthreads();
    }
}

// ---- NTT bins ----------------------------------------------------------------------
// residues out[(q * m + i) * N + j] for product i of the bin (operand `which`)
__global__ void bin_split_kernel(uint64_t* __restrict__ out, const DevDesc* __restrict__ d,
                                 const uint32_t* __restrict__ idx, size_t m, int k, int which, uint64_t p0,
                                 uint64_t p1, uint64_t p2)
{
    const size_t N = (size_t)1 << k;
    const size_t total = m * N;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < total; g += (size_t)gridDim.x * blockDim.x) {
        const size_t i = g >> k, j = g & (N - 1);
        const DevDesc D = d[idx[i]];
        const uint32_t* x = which ? D.b : D.a;
        const uint32_t n = which ? D.nb : D.na;
        uint64_t v = 0;
        if (2 * j < n) {
            v = x[2 * j];
            if (2 * j + 1 < n) v |= (uint64_t)x[2 * j + 1] << 32;
        }
        out[(0 * m + i) * N + j] = piece_to_strict(v, p0);
        out[(1 * m + i) * N + j] = piece_to_strict(v, p1);
        out[(2 * m + i) * N + j] = piece_to_strict(v, p2);
    }
}

__global__ void bin_lengths_kernel(const DevDesc* __restrict__ d, const uint32_t* __restrict__ idx, size_t m,
                                   uint32_t* zl)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
        const DevDesc D = d[idx[i]];
        zl[i] = D.na + D.nb;
    }
}

__global__ void bin_scatter_kernel(const uint32_t* __restrict__ zt, uint32_t zcap, const DevDesc* __restrict__ d,
                                   const uint32_t* __restrict__ idx, size_t m)
{
    for (size_t i = blockIdx.x; i < m; i += gridDim.x) {
        const DevDesc D = d[idx[i]];
        const uint32_t zw = D.na + D.nb;
        for (uint32_t w = threadIdx.x; w < zw; w += blockDim.x) D.z[w] = zt[i * (size_t)zcap + w];
    }
}

// ---- plans and graphs ----------------------------------------------------------------
namespace {
struct Bin {
    int k;
    uint32_t zcap;
    std::vector<uint32_t> idx;  // descriptor indices
    DevBuf<uint32_t> didx;
};

struct Plan {
    size_t count = 0;
    std::vector<uint32_t> sizes;  // na, nb pairs (the signature)
    DevBuf<DevDesc> desc;
    DevDesc* host_desc = nullptr;  // pinned staging
    std::vector<uint32_t> school;  // descriptor indices, longest first
    DevBuf<uint32_t> dschool;
    DevBuf<uint32_t> counter;
    uint32_t school_max_zw = 0;
    std::vector<Bin> bins;
    cudaGraphExec_t exec = nullptr;
    uint64_t kernels = 0;
    ~Plan()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (host_desc) cudaFreeHost(host_desc);
    }
};

std::mutex g_plan_lock;
std::map<std::vector<uint32_t>, std::unique_ptr<Plan>> g_plans;
bool g_use_graphs = true;
}  // namespace

void mul_batch_set_graphs(bool on) { g_use_graphs = on; }

static int batch_class(const pic_mul_desc& d, int mode)
{
    // -1: persistent schoolbook; k >= 1: three-prime NTT bin of length 2^k
    const size_t zw = d.na + d.nb;
    int m = mode == PIC_MUL_AUTO ? mul_auto_mode(d.na, d.nb) : mode;
    if (m == PIC_MUL_SCHOOL && zw <= kSchoolMaxWords) return -1;
    const size_t ncoef = (d.na + 1) / 2 + (d.nb + 1) / 2 - 1;
    int k = 1;
    while (((size_t)1 << k) < ncoef) k++;
    return k;
}

static void enqueue_plan(Plan& P, cudaStream_t s)
{
    if (!P.school.empty()) {
        PIC_CUDA(cudaMemsetAsync(P.counter.get(), 0, sizeof(uint32_t), s));
        const size_t smem = (size_t)P.school_max_zw * 16;
        if (smem > 48 * 1024)
            PIC_CUDA(cudaFuncSetAttribute(school_persistent_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
        const unsigned grid = (unsigned)std::min<size_t>(P.school.size(), 148 * 8);
        school_persistent_kernel<<<grid, kPSchThreads, smem, s>>>(P.desc.get(), P.dschool.get(),
                                                                 (uint32_t)P.school.size(), P.counter.get());
        PIC_CHECK_LAUNCH();
        count_launch();
    }
    for (Bin& B : P.bins) {
        const size_t m = B.idx.size();
        const size_t N = (size_t)1 << B.k;
        DevBuf<uint64_t> A(3 * m * N, s), Bb(3 * m * N, s);
        DevBuf<uint32_t> zt(m * (size_t)B.zcap, s), zl(m, s);
        for (int w = 0; w < 2; w++) {
            bin_split_kernel<<<grid_for(m * N, 256), 256, 0, s>>>(w ? Bb.get() : A.get(), P.desc.get(),
                                                                  B.didx.get(), m, B.k, w, kProductPrimes[0],
                                                                  kProductPrimes[1], kProductPrimes[2]);
            PIC_CHECK_LAUNCH();
            count_launch();
        }
        NttBatch bt;
        bt.stride = N;
        bt.count = (int)(3 * m);
        bt.per_prime = (int)m;
        for (int q = 0; q < 3; q++) bt.prime[q] = prime_tables(kProductPrimes[q]).dev;
        bt.data = A.get();
        ntt_forward_dif(bt, B.k, s);
        NttBatch bb = bt;
        bb.data = Bb.get();
        ntt_forward_dif(bb, B.k, s);
        ntt_pointwise_mont(bt, Bb.get(), B.k, s);
        ntt_inverse_dit(bt, B.k, s);
        bin_lengths_kernel<<<grid_for(m, 256), 256, 0, s>>>(P.desc.get(), B.didx.get(), m, zl.get());
        PIC_CHECK_LAUNCH();
        count_launch();
        ntt3_batch_to_words(A.get(), N, m * N, m, B.k, zt.get(), B.zcap, zl.get(), s);
        bin_scatter_kernel<<<(unsigned)std::min<size_t>(m, 148 * 16), 256, 0, s>>>(zt.get(), B.zcap, P.desc.get(),
                                                                                  B.didx.get(), m);
        PIC_CHECK_LAUNCH();
        count_launch();
    }
}

static std::unique_ptr<Plan> build_plan(const pic_mul_desc* d, size_t count, int mode, cudaStream_t s,
                                        const std::vector<uint32_t>& sig)
{
    auto P = std::make_unique<Plan>();
    P->count = count;
    P->sizes = sig;
    P->desc = DevBuf<DevDesc>(count, s);
    PIC_CUDA(cudaMallocHost((void**)&P->host_desc, sizeof(DevDesc) * count));
    ctx().alloc_calls.fetch_add(1);
    P->counter = DevBuf<uint32_t>(1, s);
    std::map<int, Bin> bins;
    for (size_t i = 0; i < count; i++) {
        const int c = batch_class(d[i], mode);
        if (c < 0) {
            P->school.push_back((uint32_t)i);
            P->school_max_zw = std::max<uint32_t>(P->school_max_zw, (uint32_t)(d[i].na + d[i].nb));
        } else {
            Bin& B = bins[c];
            B.k = c;
            B.zcap = std::max<uint32_t>(B.zcap, (uint32_t)(d[i].na + d[i].nb));
            B.idx.push_back((uint32_t)i);
        }
    }
    std::sort(P->school.begin(), P->school.end(),
              [&](uint32_t x, uint32_t y) { return d[x].na + d[x].nb > d[y].na + d[y].nb; });
    if (!P->school.empty()) {
        P->dschool = DevBuf<uint32_t>(P->school.size(), s);
        PIC_CUDA(cudaMemcpyAsync(P->dschool.get(), P->school.data(), 4 * P->school.size(), cudaMemcpyHostToDevice,
                                 s));
    }
    for (auto& kv : bins) {
        Bin& B = kv.second;
        B.didx = DevBuf<uint32_t>(B.idx.size(), s);
        PIC_CUDA(cudaMemcpyAsync(B.didx.get(), B.idx.data(), 4 * B.idx.size(), cudaMemcpyHostToDevice, s));
        P->bins.push_back(std::move(B));
    }
    for (int q = 0; q < 3; q++) prime_tables(kProductPrimes[q]);  // tables exist before any capture
    PIC_CUDA(cudaStreamSynchronize(s));
    return P;
}

void mul_batch(const pic_mul_desc* d, size_t count, int mode, cudaStream_t s)
{
    count_products(count);
    if (count == 0) return;
    std::vector<uint32_t> sig;
    sig.reserve(2 * count + 1);
    sig.push_back((uint32_t)mode);
    for (size_t i = 0; i < count; i++) {
        PIC_REQUIRE(d[i].z && d[i].a && d[i].b && d[i].na && d[i].nb, PIC_ERR_INVALID, "bad product descriptor");
        PIC_REQUIRE(d[i].na < (1ull << 31) && d[i].nb < (1ull << 31), PIC_ERR_INVALID, "operand too long");
        sig.push_back((uint32_t)d[i].na);
        sig.push_back((uint32_t)d[i].nb);
    }
    if (mode == PIC_MUL_NTT_REF || mode == PIC_MUL_FFT) {  // forms without a batched kernel
        for (size_t i = 0; i < count; i++) mul_dispatch(d[i].z, d[i].a, (size_t)d[i].na, d[i].b, (size_t)d[i].nb, mode, s);
        return;
    }
    std::lock_guard<std::mutex> g(g_plan_lock);
    auto it = g_plans.find(sig);
    if (it == g_plans.end()) {
        if (g_plans.size() >= 8) g_plans.clear();
        it = g_plans.emplace(sig, build_plan(d, count, mode, s, sig)).first;
    }
    Plan& P = *it->second;
    for (size_t i = 0; i < count; i++)
        P.host_desc[i] = DevDesc{d[i].z, d[i].a, d[i].b, (uint32_t)d[i].na, (uint32_t)d[i].nb};
    PIC_CUDA(cudaMemcpyAsync(P.desc.get(), P.host_desc, sizeof(DevDesc) * count, cudaMemcpyHostToDevice, s));
    if (!g_use_graphs) {
        enqueue_plan(P, s);
        PIC_CUDA(cudaStreamSynchronize(s));  // the pinned staging is reused by the next call
        return;
    }
    if (!P.exec) {
        cudaStream_t cs;
        PIC_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        PIC_CUDA(cudaStreamSynchronize(s));
        cudaGraph_t graph;
        PIC_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        const uint64_t before = ctx().launches.load();
        try {
            enqueue_plan(P, cs);
        } catch (...) {
            cudaStreamEndCapture(cs, &graph);
            cudaStreamDestroy(cs);
            throw;
        }
        // launches are counted when the graph runs, not when it is recorded
        P.kernels = ctx().launches.load() - before;
        ctx().launches.fetch_sub(P.kernels);
        PIC_CUDA(cudaStreamEndCapture(cs, &graph));
        PIC_CUDA(cudaGraphInstantiate(&P.exec, graph, 0));
        PIC_CUDA(cudaGraphDestroy(graph));
        PIC_CUDA(cudaStreamDestroy(cs));
    }
    PIC_CUDA(cudaGraphLaunch(P.exec, s));
    count_launch(P.kernels);
    PIC_CUDA(cudaStreamSynchronize(s));  // the pinned staging is reused by the next call
}

}  // namespace pic
