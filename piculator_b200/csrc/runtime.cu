// Context, memory and error plumbing (see common.cuh).
#include <stdio.h>
#include <string.h>

#include <stdlib.h>

#include <chrono>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace pic {

static Context g_ctx;
static std::atomic<bool> g_init{false};
static thread_local std::string t_last_error;

void set_last_error(const std::string& s) { t_last_error = s; }
const std::string& last_error() { return t_last_error; }

void throw_cuda(cudaError_t e, const char* what, const char* file, int line)
{
    char buf[512];
    snprintf(buf, sizeof buf, "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
    if (e == cudaErrorMemoryAllocation) throw Error(PIC_ERR_NO_MEMORY, buf);
    throw Error(PIC_ERR_CUDA, buf);
}

Context& ctx() { return g_ctx; }
bool initialized() { return g_init.load(); }

void require_init()
{
    if (!g_init.load()) throw Error(PIC_ERR_NOT_INITIALIZED, "pic_init has not been called");
}

cudaStream_t resolve(pic_stream s) { return s ? (cudaStream_t)s : g_ctx.stream; }

void init_context(int device)
{
    std::lock_guard<std::recursive_mutex> g(g_ctx.lock);
    if (g_init.load()) {
        PIC_REQUIRE(device == g_ctx.device, PIC_ERR_INVALID,
                    "pic_init: library already initialised on another device");
        return;
    }
    int n = 0;
    PIC_CUDA(cudaGetDeviceCount(&n));
    PIC_REQUIRE(device >= 0 && device < n, PIC_ERR_INVALID, "pic_init: no such device");
    PIC_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    PIC_CUDA(cudaGetDeviceProperties(&prop, device));
    PIC_REQUIRE(prop.major == 10, PIC_ERR_CUDA,
                "pic_init: this build targets sm_100a (B200); device is " + std::string(prop.name));
    g_ctx.device = device;
    g_ctx.num_sms = prop.multiProcessorCount;
    PIC_CUDA(cudaStreamCreateWithFlags(&g_ctx.stream, cudaStreamNonBlocking));
    cudaMemPool_t pool;
    PIC_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t thr = UINT64_MAX;
    PIC_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    // every buffer lives on one stream, where reuse in stream order needs no
    // opportunistic reuse; without it the pool's choice of block does not
    // depend on how far the GPU has got, so repeated calls get the same
    // placement
    int no = 0;
    PIC_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowOpportunistic, &no));
    g_ctx.pinned_words_cap = 1 << 16;
    PIC_CUDA(cudaMallocHost((void**)&g_ctx.pinned_words, g_ctx.pinned_words_cap * sizeof(uint32_t)));
    g_init.store(true);
}

void shutdown_context()
{
    std::lock_guard<std::recursive_mutex> g(g_ctx.lock);
    if (!g_init.load()) return;
    workspace_release_all();
    cudaStreamSynchronize(g_ctx.stream);
    // hand the pool's unused memory back to the device (buffers other
    // threads still hold keep theirs)
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, g_ctx.device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
    if (g_ctx.pinned_words) cudaFreeHost(g_ctx.pinned_words);
    g_ctx.pinned_words = nullptr;
    cudaStreamDestroy(g_ctx.stream);
    g_ctx.stream = nullptr;
    g_init.store(false);
}

bool timeline_on();

// host time spent in the allocator (timeline diagnostics)
namespace {
struct AllocStat {
    double total_ms = 0, max_ms = 0;
    size_t calls = 0, max_bytes = 0;
};
AllocStat g_alloc_stat;
}  // namespace

static void alloc_stat(double ms, size_t bytes)
{
    g_alloc_stat.total_ms += ms;
    g_alloc_stat.calls++;
    if (ms > g_alloc_stat.max_ms) {
        g_alloc_stat.max_ms = ms;
        g_alloc_stat.max_bytes = bytes;
    }
}

void* dev_alloc(size_t bytes, cudaStream_t s)
{
    int f = g_ctx.fail_allocs.load();
    while (f > 0) {
        if (g_ctx.fail_allocs.compare_exchange_weak(f, f - 1))
            throw Error(PIC_ERR_NO_MEMORY, "device allocation failed (injected)");
    }
    void* p = nullptr;
    const bool tl = timeline_on();
    const auto t0 = tl ? std::chrono::steady_clock::now() : std::chrono::steady_clock::time_point();
    cudaError_t e = cudaMallocAsync(&p, bytes, s);
    if (tl) alloc_stat(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count(), bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        char buf[256];
        snprintf(buf, sizeof buf, "cudaMallocAsync(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
        throw Error(PIC_ERR_NO_MEMORY, buf);
    }
    g_ctx.bytes_in_use.fetch_add(bytes);
    g_ctx.alloc_calls.fetch_add(1);
    return p;
}

cudaError_t raw_dev_alloc(void** p, size_t bytes)
{
    const cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return e;
    }
    g_ctx.alloc_calls.fetch_add(1);
    return e;
}

size_t device_available_bytes()
{
    size_t free_b = 0, total_b = 0;
    PIC_CUDA(cudaMemGetInfo(&free_b, &total_b));
    // memory the stream-ordered pool holds but no live buffer uses is available too
    cudaMemPool_t pool;
    PIC_CUDA(cudaDeviceGetDefaultMemPool(&pool, g_ctx.device));
    uint64_t reserved = 0;
    PIC_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved));
    const uint64_t used = g_ctx.bytes_in_use.load();
    return free_b + (reserved > used ? (size_t)(reserved - used) : 0);
}

void reserve_pool(size_t bytes, cudaStream_t s)
{
    cudaMemPool_t pool;
    PIC_CUDA(cudaDeviceGetDefaultMemPool(&pool, g_ctx.device));
    uint64_t reserved = 0;
    PIC_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved));
    if (reserved >= bytes) return;
    const uint64_t used = g_ctx.bytes_in_use.load();
    size_t free_b = 0, total_b = 0;
    PIC_CUDA(cudaMemGetInfo(&free_b, &total_b));
    size_t want = bytes - (size_t)(used < reserved ? used : reserved);
    const size_t cap = free_b / 10 * 9 + (size_t)(reserved > used ? reserved - used : 0);
    if (want > cap) want = cap;
    if (want == 0) return;
    void* p = nullptr;
    if (cudaMallocAsync(&p, want, s) != cudaSuccess) {
        cudaGetLastError();  // no room for one block that size: allocate as needed instead
        return;
    }
    g_ctx.alloc_calls.fetch_add(1);
    PIC_CUDA(cudaFreeAsync(p, s));
    PIC_CUDA(cudaStreamSynchronize(s));
}

namespace {
struct Workspace {
    std::mutex lock;
    void* ptr = nullptr;
    size_t bytes = 0;
    bool leased = false;
};
Workspace g_ws;
}  // namespace

WorkspaceLease::WorkspaceLease(size_t bytes, cudaStream_t s)
{
    if (s != g_ctx.stream || bytes == 0) return;
    std::lock_guard<std::mutex> g(g_ws.lock);
    if (g_ws.leased) return;
    if (g_ws.bytes < bytes) {
        if (g_ws.ptr) dev_free(g_ws.ptr, g_ws.bytes, s);  // stream-ordered: earlier users finish first
        g_ws.ptr = nullptr;
        g_ws.bytes = 0;
        g_ws.ptr = dev_alloc(bytes, s);  // throws on no memory, with nothing leased
        g_ws.bytes = bytes;
    }
    g_ws.leased = true;
    ptr = g_ws.ptr;
}

WorkspaceLease::~WorkspaceLease()
{
    if (!ptr) return;
    std::lock_guard<std::mutex> g(g_ws.lock);
    g_ws.leased = false;
}

void workspace_release_all()
{
    std::lock_guard<std::mutex> g(g_ws.lock);
    if (g_ws.ptr && !g_ws.leased) {
        dev_free(g_ws.ptr, g_ws.bytes, g_ctx.stream);
        g_ws.ptr = nullptr;
        g_ws.bytes = 0;
    }
}

void dev_free(void* p, size_t bytes, cudaStream_t s)
{
    if (!p) return;
    const bool tl = timeline_on();
    const auto t0 = tl ? std::chrono::steady_clock::now() : std::chrono::steady_clock::time_point();
    cudaFreeAsync(p, s);
    if (tl) alloc_stat(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count(), 0);
    g_ctx.bytes_in_use.fetch_sub(bytes);
}

void read_words(uint32_t* host, const uint32_t* dev, size_t count, cudaStream_t s)
{
    if (count == 0) return;
    if (count <= g_ctx.pinned_words_cap) {
        std::lock_guard<std::recursive_mutex> g(g_ctx.lock);
        PIC_CUDA(cudaMemcpyAsync(g_ctx.pinned_words, dev, count * sizeof(uint32_t),
                                 cudaMemcpyDeviceToHost, s));
        PIC_CUDA(cudaStreamSynchronize(s));
        memcpy(host, g_ctx.pinned_words, count * sizeof(uint32_t));
    } else {
        PIC_CUDA(cudaMemcpyAsync(host, dev, count * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        PIC_CUDA(cudaStreamSynchronize(s));
    }
}

// ---- tracing ---------------------------------------------------------------------
bool tracing()
{
    static const bool on = getenv("PIC_TRACE") != nullptr;
    return on;
}

TraceSpan::TraceSpan(cudaStream_t st) : s(st)
{
    if (!tracing()) return;
    PIC_CUDA(cudaEventCreate(&a));
    PIC_CUDA(cudaEventCreate(&b));
    PIC_CUDA(cudaEventRecord(a, s));
}

double TraceSpan::end_ms()
{
    if (!a) return 0.0;
    PIC_CUDA(cudaEventRecord(b, s));
    PIC_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    PIC_CUDA(cudaEventElapsedTime(&ms, a, b));
    return ms;
}

TraceSpan::~TraceSpan()
{
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
}

// ---- timeline: stream-ordered events, no synchronisation until the dump -------
namespace {
struct TimelineMark {
    const char* tag;
    cudaEvent_t e;
    int k;
};
std::vector<TimelineMark> g_timeline;
std::mutex g_timeline_lock;
}  // namespace

bool timeline_on()
{
    static const bool on = getenv("PIC_TIMELINE") != nullptr;
    return on;
}

void timeline_mark(const char* tag, cudaStream_t s, int k)
{
    if (!timeline_on()) return;
    TimelineMark m{tag, nullptr, k};
    PIC_CUDA(cudaEventCreate(&m.e));
    PIC_CUDA(cudaEventRecord(m.e, s));
    std::lock_guard<std::mutex> g(g_timeline_lock);
    g_timeline.push_back(m);
}

void timeline_dump()
{
    if (!timeline_on()) return;
    std::lock_guard<std::mutex> g(g_timeline_lock);
    if (g_timeline.empty()) return;
    PIC_CUDA(cudaEventSynchronize(g_timeline.back().e));
    for (size_t i = 1; i < g_timeline.size(); i++) {
        float ms = 0;
        PIC_CUDA(cudaEventElapsedTime(&ms, g_timeline[i - 1].e, g_timeline[i].e));
        if (g_timeline[i].k >= 0)
            fprintf(stderr, "{\"timeline\": \"%s\", \"k\": %d, \"ms\": %.3f}\n", g_timeline[i].tag, g_timeline[i].k,
                    ms);
        else
            fprintf(stderr, "{\"timeline\": \"%s\", \"ms\": %.3f}\n", g_timeline[i].tag, ms);
    }
    for (auto& m : g_timeline) cudaEventDestroy(m.e);
    g_timeline.clear();
    fprintf(stderr, "{\"timeline_alloc\": {\"calls\": %zu, \"total_ms\": %.3f, \"max_ms\": %.3f, \"max_bytes\": %zu}}\n",
            g_alloc_stat.calls, g_alloc_stat.total_ms, g_alloc_stat.max_ms, g_alloc_stat.max_bytes);
    g_alloc_stat = AllocStat();
}

void trace_point(const char* tag, cudaStream_t s)
{
    if (!tracing()) return;
    PIC_CUDA(cudaStreamSynchronize(s));
    static const auto t0 = std::chrono::steady_clock::now();
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    cudaMemPool_t pool;
    PIC_CUDA(cudaDeviceGetDefaultMemPool(&pool, g_ctx.device));
    uint64_t reserved = 0, used_pool = 0;
    PIC_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved));
    PIC_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used_pool));
    fprintf(stderr, "{\"trace\": \"point\", \"tag\": \"%s\", \"host_ms\": %.3f, \"pool_reserved_gb\": %.3f, "
            "\"pool_used_gb\": %.3f}\n", tag, ms, reserved / 1e9, used_pool / 1e9);
}

// ---- live kernel timing ------------------------------------------------------
namespace {
struct ProfRec {
    int cls;
    double bytes;
    cudaEvent_t a, b;
};
std::mutex g_prof_lock;
std::atomic<bool> g_prof_on{false};
std::vector<ProfRec> g_prof;
std::vector<cudaEvent_t> g_ev_pool;
cudaEvent_t take_event()
{
    if (g_ev_pool.empty()) {
        cudaEvent_t e;
        PIC_CUDA(cudaEventCreate(&e));
        return e;
    }
    cudaEvent_t e = g_ev_pool.back();
    g_ev_pool.pop_back();
    return e;
}
}  // namespace

const char* kernel_class_name(int c)
{
    static const char* names[KC_COUNT] = {"ntt_cols", "ntt_rows", "ntt_pointwise", "split", "crt_carry",
                                          "carry_scan", "linear", "schoolbook", "fft_cols", "fft_rows",
                                          "bsr_level", "other"};
    return (c >= 0 && c < KC_COUNT) ? names[c] : "?";
}

bool profiling() { return g_prof_on.load(std::memory_order_relaxed); }

ProfScope::ProfScope(KernelClass c, double bytes, cudaStream_t st) : s(st)
{
    if (!profiling()) return;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone) return;
    std::lock_guard<std::mutex> g(g_prof_lock);
    ProfRec r{(int)c, bytes, take_event(), take_event()};
    PIC_CUDA(cudaEventRecord(r.a, st));
    slot = (int)g_prof.size();
    g_prof.push_back(r);
}

ProfScope::~ProfScope()
{
    if (slot < 0) return;
    std::lock_guard<std::mutex> g(g_prof_lock);
    cudaEventRecord(g_prof[slot].b, s);
}

void profile_begin()
{
    std::lock_guard<std::mutex> g(g_prof_lock);
    for (auto& r : g_prof) {
        g_ev_pool.push_back(r.a);
        g_ev_pool.push_back(r.b);
    }
    g_prof.clear();
    g_prof_on.store(true);
}

int profile_end(pic_kernel_stat* out, int cap)
{
    g_prof_on.store(false);
    std::lock_guard<std::mutex> g(g_prof_lock);
    pic_kernel_stat acc[KC_COUNT];
    memset(acc, 0, sizeof acc);
    for (auto& r : g_prof) {
        PIC_CUDA(cudaEventSynchronize(r.b));
        float ms = 0;
        PIC_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
        acc[r.cls].launches++;
        acc[r.cls].seconds += ms / 1000.0;
        acc[r.cls].bytes += r.bytes;
    }
    int n = 0;
    for (int c = 0; c < KC_COUNT; c++) {
        if (!acc[c].launches) continue;
        if (n < cap) {
            out[n] = acc[c];
            snprintf(out[n].name, sizeof out[n].name, "%s", kernel_class_name(c));
        }
        n++;
    }
    return n;
}

}  // namespace pic
