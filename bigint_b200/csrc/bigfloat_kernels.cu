// Digit kernels of the device-resident BigFloat steps (the reference's
// BigFloat::reciprocal, src/bigint.cpp:1044-1071, run on the GPU).
//
// Values are the reference's Digits: little-endian uint32_t digits of 28
// bits.  The kernels here are the O(n) steps between the products:
//   * frame add / subtract (BigFloat::add_or_sub, src/bigint.cpp:849-936):
//     both operands placed in one frame of L digits at digit offsets; the
//     carry (or borrow) is resolved by a three-launch scan -- per-block
//     (generate, propagate) aggregates, one block scanning the aggregates,
//     then every block applying its carry-in -- with no inter-block waits;
//   * magnitude compare of two framed operands (highest differing digit);
//   * bit shifts by 1..27 (BigFloat::shift_right / shift_left,
//     src/bigint.cpp:791-812);
//   * the nonzero extent of a digit array (highest nonzero digit and lowest
//     nonzero digit at or above two given positions), which the host reads to
//     strip leading and trailing zeros (remove_leading_zero /
//     remove_tail_zero, src/bigint.cpp:814-847, and the truncation of
//     mul_digits, include/bigint/mul.h:301-312).
#include <cuda_runtime.h>

#include <cstdint>

#include "engine.h"

namespace bgpu {
namespace {

constexpr uint32_t kMask28 = (1u << 28) - 1u;
constexpr int kAsThreads = 256;
constexpr int kAsPer = 8;  // consecutive digits per thread
constexpr uint32_t kAsBlock = kAsThreads * kAsPer;
constexpr int kScanThreads = 1024;

// Carry state of a digit run: bit 0 generate (a carry or borrow leaves the
// run whatever comes in), bit 1 propagate (an incoming one passes through).
// compose(lo, hi) is the state of lo followed by hi.
__device__ __forceinline__ uint32_t compose(uint32_t lo, uint32_t hi) {
    const uint32_t g = (hi & 1u) | ((hi >> 1) & lo & 1u);
    const uint32_t p = (hi >> 1) & (lo >> 1) & 1u;
    return g | (p << 1);
}

__device__ __forceinline__ uint32_t framed(const uint32_t* p, int64_t o, uint32_t n, uint32_t j) {
    const int64_t i = (int64_t)j - o;
    return (i >= 0 && i < (int64_t)n) ? p[i] : 0u;
}

__device__ __forceinline__ uint32_t digit_state(uint32_t x, uint32_t y, int sub) {
    if (sub) return (uint32_t)(x < y) | ((uint32_t)(x == y) << 1);
    const uint32_t t = x + y;
    return (uint32_t)(t > kMask28) | ((uint32_t)(t == kMask28) << 1);
}

// State of this thread's kAsPer digits (identity 2 = propagate, no generate).
__device__ __forceinline__ uint32_t thread_state(const FrameOp& f, uint32_t j0) {
    uint32_t s = 2u;
#pragma unroll
    for (int k = 0; k < kAsPer; ++k) {
        const uint32_t j = j0 + (uint32_t)k;
        if (j < f.L) s = compose(s, digit_state(framed(f.a, f.oa, f.na, j), framed(f.b, f.ob, f.nb, j), f.sub));
    }
    return s;
}

// Exclusive scan of the block's thread states; returns the state of all
// threads before this one (2 for thread 0) and writes the block total.
__device__ __forceinline__ uint32_t block_exclusive(uint32_t s, uint32_t* total) {
    __shared__ uint32_t s_warp[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t inc = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc = compose(v, inc);
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < nw ? s_warp[lane] : 2u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w = compose(v, w);
        }
        if (lane < nw) s_warp[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    uint32_t before = __shfl_up_sync(0xffffffffu, inc, 1);
    if (lane == 0) before = 2u;
    if (warp > 0) before = compose(s_warp[warp - 1], before);
    if (total) *total = s_warp[nw - 1];
    return before;
}

// A compare result (k_cmp) in f.order swaps the operands when B is larger.
__device__ __forceinline__ FrameOp ordered(FrameOp f) {
    if (f.order && (*f.order & 3u) == 2u) {
        const uint32_t* p = f.a;
        f.a = f.b;
        f.b = p;
        const int64_t o = f.oa;
        f.oa = f.ob;
        f.ob = o;
        const uint32_t n = f.na;
        f.na = f.nb;
        f.nb = n;
    }
    return f;
}

__global__ void __launch_bounds__(kAsThreads) k_as_aggregate(const FrameOp fin, uint32_t* agg) {
    const FrameOp f = ordered(fin);
    const uint32_t j0 = blockIdx.x * kAsBlock + threadIdx.x * kAsPer;
    uint32_t total;
    block_exclusive(thread_state(f, j0), &total);
    if (threadIdx.x == 0) agg[blockIdx.x] = total;
}

// One block: carry into every block from the block aggregates.
__global__ void __launch_bounds__(kScanThreads) k_as_scan(const uint32_t* agg, uint32_t nblk, uint32_t* cin) {
    const uint32_t per = (nblk + kScanThreads - 1) / kScanThreads;
    const uint32_t b0 = threadIdx.x * per;
    uint32_t s = 2u;
    for (uint32_t k = 0; k < per; ++k)
        if (b0 + k < nblk) s = compose(s, agg[b0 + k]);
    uint32_t before = block_exclusive(s, nullptr);
    for (uint32_t k = 0; k < per; ++k) {
        if (b0 + k >= nblk) break;
        cin[b0 + k] = before & 1u;  // carry in: generated before, none enters the frame
        before = compose(before, agg[b0 + k]);
    }
}

__global__ void __launch_bounds__(kAsThreads) k_as_apply(const FrameOp fin, const uint32_t* cin,
                                                         uint32_t* out) {
    const FrameOp f = ordered(fin);
    const uint32_t j0 = blockIdx.x * kAsBlock + threadIdx.x * kAsPer;
    const uint32_t before = block_exclusive(thread_state(f, j0), nullptr);
    const uint32_t c0 = cin[blockIdx.x];
    uint32_t c = (before & 1u) | ((before >> 1) & c0);
#pragma unroll
    for (int k = 0; k < kAsPer; ++k) {
        const uint32_t j = j0 + (uint32_t)k;
        if (j >= f.L) break;
        const uint32_t x = framed(f.a, f.oa, f.na, j), y = framed(f.b, f.ob, f.nb, j);
        if (f.sub) {
            out[j] = (x - y - c) & kMask28;
            c = (x < y + c) ? 1u : 0u;
        } else {
            const uint32_t t = x + y + c;
            out[j] = t & kMask28;
            c = t >> 28;
        }
        if (j == f.L - 1) out[f.L] = f.sub ? 0u : c;  // carry out of the frame
    }
}

// Highest frame position where the framed operands differ, packed for one
// 64-bit atomicMax: r = (j + 1) << 2 | (1 if A_j > B_j else 2); 0 when equal.
__global__ void k_cmp(const FrameOp f, unsigned long long* r) {
    unsigned long long best = 0;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < f.L; j += gridDim.x * blockDim.x) {
        const uint32_t x = framed(f.a, f.oa, f.na, j), y = framed(f.b, f.ob, f.nb, j);
        if (x != y) best = ((unsigned long long)(j + 1) << 2) | (x > y ? 1u : 2u);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long v = __shfl_xor_sync(0xffffffffu, best, o);
        best = v > best ? v : best;
    }
    if ((threadIdx.x & 31) == 0 && best) atomicMax(r, best);
}

// Nonzero extent, three keys packed for 64-bit atomicMax from a zeroed block:
// r[0] = (j + 1) << 32 | d[j] for the highest nonzero j; r[1], r[2] =
// 2^32 - j for the lowest nonzero j >= from0, from1.
__global__ void k_extent(const uint32_t* d, uint32_t n, uint32_t from0, uint32_t from1,
                         unsigned long long* r) {
    unsigned long long hi = 0, lo0 = 0, lo1 = 0;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const uint32_t v = d[j];
        if (v == 0) continue;
        hi = ((unsigned long long)(j + 1) << 32) | v;  // j grows along the loop
        const unsigned long long key = (1ull << 32) - j;
        if (j >= from0 && key > lo0) lo0 = key;
        if (j >= from1 && key > lo1) lo1 = key;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long v = __shfl_xor_sync(0xffffffffu, hi, o);
        hi = v > hi ? v : hi;
        v = __shfl_xor_sync(0xffffffffu, lo0, o);
        lo0 = v > lo0 ? v : lo0;
        v = __shfl_xor_sync(0xffffffffu, lo1, o);
        lo1 = v > lo1 ? v : lo1;
    }
    if ((threadIdx.x & 31) == 0) {
        if (hi) atomicMax(r, hi);
        if (lo0) atomicMax(r + 1, lo0);
        if (lo1) atomicMax(r + 2, lo1);
    }
}

__global__ void k_shift_right(const uint32_t* v, uint32_t n, uint32_t s, uint32_t* out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t hi = i + 1 < n ? v[i + 1] << (28u - s) : 0u;
        out[i] = ((v[i] >> s) | hi) & kMask28;
    }
}

__global__ void k_shift_left(const uint32_t* v, uint32_t n, uint32_t s, uint32_t* out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x) {
        const uint32_t cur = i < n ? v[i] << s : 0u;
        const uint32_t lo = i > 0 ? v[i - 1] >> (28u - s) : 0u;
        out[i] = (cur | lo) & kMask28;
    }
}

uint32_t grid_for(uint64_t n, uint32_t threads) {
    const uint64_t b = (n + threads - 1) / threads;
    return (uint32_t)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

}  // namespace

uint32_t frame_blocks(uint32_t L) { return (L + kAsBlock - 1) / kAsBlock; }

cudaError_t launch_frame_addsub(const FrameOp& f, uint32_t* agg, uint32_t* cin, uint32_t* out,
                                cudaStream_t st) {
    const uint32_t nblk = frame_blocks(f.L);
    k_as_aggregate<<<nblk, kAsThreads, 0, st>>>(f, agg);
    k_as_scan<<<1, kScanThreads, 0, st>>>(agg, nblk, cin);
    k_as_apply<<<nblk, kAsThreads, 0, st>>>(f, cin, out);
    return cudaGetLastError();
}

cudaError_t launch_frame_cmp(const FrameOp& f, unsigned long long* r, cudaStream_t st) {
    k_cmp<<<grid_for(f.L, 256), 256, 0, st>>>(f, r);
    return cudaGetLastError();
}

cudaError_t launch_extent(const uint32_t* d, uint32_t n, uint32_t from0, uint32_t from1,
                          unsigned long long* r, cudaStream_t st) {
    k_extent<<<grid_for(n, 256), 256, 0, st>>>(d, n, from0, from1, r);
    return cudaGetLastError();
}

cudaError_t launch_shift_digits(const uint32_t* v, uint32_t n, uint32_t s, bool left, uint32_t* out,
                                cudaStream_t st) {
    if (left)
        k_shift_left<<<grid_for((uint64_t)n + 1, 256), 256, 0, st>>>(v, n, s, out);
    else
        k_shift_right<<<grid_for(n, 256), 256, 0, st>>>(v, n, s, out);
    return cudaGetLastError();
}

}  // namespace bgpu
