// Carry (and borrow) resolution over long word arrays.
//
// Every linear step of the path -- the product's coefficient-to-word
// conversion (ntt_to_int NTT.cpp:343-369, fft_to_int FFT.cpp:520-571), uadd /
// usub (BigFloat.cpp:184-287) and mul(uint32) (BigFloat.cpp:156-183) -- is a
// sequential carry loop in the reference.  Here each word first gets a raw
// digit d_i and a "generate" bit g_i (carry out no matter what comes in); the
// carry into word i is then the carry-lookahead prefix
//     c_(i+1) = g_i | (p_i & c_i),   p_i = (d_i == all-ones)   [add]
//     b_(i+1) = g_i | (p_i & b_i),   p_i = (d_i == 0)          [subtract]
// which is associative, so it runs as a block scan inside each CTA plus a
// reduce-then-scan across CTAs (no inter-CTA waiting, no spin loops):
//   K1  raw digits -> in-block resolved words + one (G, P) per CTA
//   K2  one CTA scans the per-CTA pairs -> carry-in per CTA + final carry
//   K3  CTAs with carry-in 1 ripple it through their own words.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pic {

// (g, p) packed as bit0 = generate, bit1 = propagate.  Identity = propagate.
constexpr uint32_t kGPIdentity = 2u;

__device__ __forceinline__ uint32_t gp_combine(uint32_t lo, uint32_t hi)
{
    const uint32_t g = (hi & 1u) | ((hi >> 1) & lo & 1u);
    const uint32_t p = (hi >> 1) & (lo >> 1) & 1u;
    return g | (p << 1);
}

// Exclusive block scan of one (g, p) per thread, threads in position order.
// Returns the exclusive prefix; *total receives the block aggregate.  Must be
// called by every thread of the block (blockDim.x a multiple of 32, <= 1024).
__device__ __forceinline__ uint32_t block_gp_scan(uint32_t gp, uint32_t* total)
{
    __shared__ uint32_t s_warp[32];
    __shared__ uint32_t s_tot;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    uint32_t v = gp;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        uint32_t o = __shfl_up_sync(0xffffffffu, v, off);
        if (lane >= off) v = gp_combine(o, v);
    }
    uint32_t excl = __shfl_up_sync(0xffffffffu, v, 1);
    if (lane == 0) excl = kGPIdentity;
    if (lane == 31) s_warp[wid] = v;
    __syncthreads();
    if (wid == 0) {
        uint32_t w = lane < nw ? s_warp[lane] : kGPIdentity;
        uint32_t iv = w;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            uint32_t o = __shfl_up_sync(0xffffffffu, iv, off);
            if (lane >= off) iv = gp_combine(o, iv);
        }
        uint32_t ex = __shfl_up_sync(0xffffffffu, iv, 1);
        if (lane == 0) ex = kGPIdentity;
        if (lane == 31) s_tot = iv;
        __syncwarp();
        s_warp[lane] = ex;
    }
    __syncthreads();
    const uint32_t res = gp_combine(s_warp[wid], excl);
    const uint32_t tot = s_tot;
    __syncthreads();
    *total = tot;
    return res;
}

// Warp-reduced max / min: one shared or global atomic per warp instead of one
// per qualifying element (a single hot address serialises per-element atomics).
__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v)
{
#pragma unroll
    for (int off = 16; off; off >>= 1) {
        const unsigned long long o = __shfl_xor_sync(0xffffffffu, v, off);
        v = o > v ? o : v;
    }
    return v;
}

__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v)
{
#pragma unroll
    for (int off = 16; off; off >>= 1) {
        const unsigned long long o = __shfl_xor_sync(0xffffffffu, v, off);
        v = o < v ? o : v;
    }
    return v;
}

// Block-wide max of one value per thread (all threads call; blockDim % 32 == 0).
__device__ __forceinline__ unsigned long long block_max_u64(unsigned long long v)
{
    __shared__ unsigned long long s_m;
    if (threadIdx.x == 0) s_m = 0;
    __syncthreads();
    v = warp_max_u64(v);
    if ((threadIdx.x & 31) == 0 && v) atomicMax(&s_m, v);
    __syncthreads();
    const unsigned long long r = s_m;
    __syncthreads();
    return r;
}

__device__ __forceinline__ unsigned long long block_min_u64(unsigned long long v)
{
    __shared__ unsigned long long s_m;
    if (threadIdx.x == 0) s_m = ~0ull;
    __syncthreads();
    v = warp_min_u64(v);
    if ((threadIdx.x & 31) == 0 && v != ~0ull) atomicMin(&s_m, v);
    __syncthreads();
    const unsigned long long r = s_m;
    __syncthreads();
    return r;
}

enum CarryMode { kCarryAdd = 0, kCarrySub = 1 };

// Cross-CTA phases (carry.cu).  agg[c] = (G, P) of CTA c; words_per_cta words
// per CTA; K3 also needs the array length.
void carry_scan_aggregates(uint32_t* agg, size_t nctas, uint32_t* final_carry, cudaStream_t s);
void carry_ripple(uint32_t* z, size_t nwords, size_t words_per_cta, const uint32_t* agg_cin,
                  size_t nctas, CarryMode mode, cudaStream_t s);

// Segmented forms for batches of products: `count` segments of `cpp` CTAs;
// product i writes zlen[i] words at z + i * zcap.
void carry_scan_segments(uint32_t* agg, size_t count, size_t cpp, cudaStream_t s);
void carry_ripple_batch(uint32_t* z, uint32_t zcap, const uint32_t* zlen, size_t words_per_cta,
                        const uint32_t* agg_cin, size_t count, size_t cpp, cudaStream_t s);

}  // namespace pic
