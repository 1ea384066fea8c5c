// Runtime plumbing shared by every translation unit of libpiculator_b200:
// errors (C++ exceptions internally, pic_status at the C ABI), the device
// context (one library stream per process), stream-ordered device buffers,
// and small pinned-host staging for device->host metadata reads.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <mutex>
#include <stdexcept>
#include <string>

#include "piculator_b200.h"

namespace pic {

struct Error : std::runtime_error {
    pic_status status;
    Error(pic_status s, const std::string& msg) : std::runtime_error(msg), status(s) {}
};

[[noreturn]] void throw_cuda(cudaError_t e, const char* what, const char* file, int line);

#define PIC_CUDA(call)                                                     \
    do {                                                                   \
        cudaError_t _e = (call);                                           \
        if (_e != cudaSuccess) ::pic::throw_cuda(_e, #call, __FILE__, __LINE__); \
    } while (0)

#define PIC_CHECK_LAUNCH() PIC_CUDA(cudaGetLastError())

#define PIC_REQUIRE(cond, status, msg)                 \
    do {                                               \
        if (!(cond)) throw ::pic::Error((status), (msg)); \
    } while (0)

// ---- context ---------------------------------------------------------------
struct Context {
    int device = -1;
    cudaStream_t stream = nullptr;       // the library's stream
    int num_sms = 0;
    std::recursive_mutex lock;           // host-side bookkeeping
    std::atomic<uint64_t> launches{0};   // kernel launches issued by the library
    std::atomic<uint64_t> bytes_in_use{0};
    std::atomic<int> fail_allocs{0};     // fault-injection hook
    std::atomic<uint64_t> alloc_calls{0};  // device allocations made (pool and direct)
    std::atomic<uint64_t> products{0};     // multi-word products formed (any kernel)
    std::atomic<uint64_t> fft_recomputes{0};  // FFT products redone with the NTT
    uint32_t* pinned_words = nullptr;    // small pinned staging for metadata reads
    size_t pinned_words_cap = 0;
};

Context& ctx();
bool initialized();
void require_init();
cudaStream_t resolve(pic_stream s);

inline void count_launch(uint64_t n = 1) { ctx().launches.fetch_add(n, std::memory_order_relaxed); }
inline void count_products(uint64_t n) { ctx().products.fetch_add(n, std::memory_order_relaxed); }

// ---- device memory -----------------------------------------------------------
// Stream-ordered allocations from the device's default memory pool (release
// threshold raised at init so freed blocks stay cached for reuse).
void* dev_alloc(size_t bytes, cudaStream_t s);
// cudaMalloc for the long-lived tables (twiddles), counted with the pool
// allocations; returns cudaSuccess or the error, which it clears.
cudaError_t raw_dev_alloc(void** p, size_t bytes);
void dev_free(void* p, size_t bytes, cudaStream_t s);
// Free device memory plus what the allocation pool holds unused.
size_t device_available_bytes();
// Grows the stream-ordered pool (which never releases memory) to hold at
// least `bytes` as one free block, so that a computation whose peak fits in
// it never grows the pool in the middle: growth maps and clears new physical
// memory while the GPU may be idle, a pause of up to some hundred ms.
// Capped at 90 % of what the device has left.
void reserve_pool(size_t bytes, cudaStream_t s);

// A grow-only device workspace on the context's stream, kept between calls:
// the work arrays of the largest transforms always land at the same
// addresses.  (Blocks of several GB placed afresh by the pool on every call
// made the same kernels run up to 40 % slower on some calls.)  lease() returns
// nullptr when `s` is not the context's stream or the workspace is already
// leased; the caller then allocates as usual.  The lease ends with the object.
struct WorkspaceLease {
    void* ptr = nullptr;
    WorkspaceLease(size_t bytes, cudaStream_t s);
    ~WorkspaceLease();
    WorkspaceLease(const WorkspaceLease&) = delete;
    WorkspaceLease& operator=(const WorkspaceLease&) = delete;
};
void workspace_release_all();  // frees the workspace (pic_shutdown)

template <typename T>
struct DevBuf {
    T* ptr = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    DevBuf() = default;
    DevBuf(size_t count, cudaStream_t st) : n(count), s(st)
    {
        ptr = (T*)dev_alloc(sizeof(T) * (count ? count : 1), st);
    }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : ptr(o.ptr), n(o.n), s(o.s) { o.ptr = nullptr; o.n = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept
    {
        if (this != &o) {
            reset();
            ptr = o.ptr; n = o.n; s = o.s;
            o.ptr = nullptr; o.n = 0;
        }
        return *this;
    }
    ~DevBuf() { reset(); }
    void reset()
    {
        if (ptr) dev_free(ptr, sizeof(T) * (n ? n : 1), s);
        ptr = nullptr;
        n = 0;
    }
    T* get() const { return ptr; }
};

// Reads `count` words from device memory (stream-ordered, then synchronises).
void read_words(uint32_t* host, const uint32_t* dev, size_t count, cudaStream_t s);

// ---- live kernel timing -------------------------------------------------------
// When enabled (pic_profile_begin), each instrumented launch is bracketed by a
// pair of CUDA events on its own stream and credited with the algorithmic
// bytes it must move; pic_profile_end reduces them per kernel class.
enum KernelClass {
    KC_NTT_COLS = 0, KC_NTT_ROWS, KC_NTT_POINTWISE, KC_SPLIT, KC_CRT, KC_CARRY, KC_LINEAR, KC_SCHOOL,
    KC_FFT_COLS, KC_FFT_ROWS, KC_BSR, KC_OTHER, KC_COUNT
};
const char* kernel_class_name(int c);
bool profiling();
struct ProfScope {
    int slot = -1;
    cudaStream_t s = nullptr;
    ProfScope(KernelClass c, double bytes, cudaStream_t st);
    ~ProfScope();
};

// Tracing: when the environment variable PIC_TRACE is set, phases print one
// JSON line each to stderr with their device time.
bool tracing();
// With tracing on: synchronise `s` and print host time and pool occupancy.
void trace_point(const char* tag, cudaStream_t s);
// With PIC_TIMELINE set: record a stream-ordered event (no synchronisation);
// timeline_dump prints the device time between consecutive marks, idle gaps
// included.
// `k` (when >= 0) is printed with the mark: the log2 transform length of the
// merges that end there.
void timeline_mark(const char* tag, cudaStream_t s, int k = -1);
void timeline_dump();
struct TraceSpan {
    cudaEvent_t a = nullptr, b = nullptr;
    cudaStream_t s = nullptr;
    TraceSpan(cudaStream_t st);
    double end_ms();  // synchronises
    ~TraceSpan();
};

inline unsigned grid_for(size_t n, unsigned block, unsigned cap = 148u * 32u)
{
    size_t g = (n + block - 1) / block;
    if (g == 0) g = 1;
    if (g > cap) g = cap;
    return (unsigned)g;
}

}  // namespace pic
