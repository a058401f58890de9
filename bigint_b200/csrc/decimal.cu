// Decimal text to binary on the device (the reference's BigInt(const
// std::string&) with convert_from_dec_string, src/bigint.cpp:25-124).
//
// The digit string is cut into leaves of 19 digits (one u64 each) from its
// least significant end, and leaves are paired level by level:
//   segment_{j+1}[p] = segment_j[2p+1] * 10^(19 * 2^j) + segment_j[2p].
// A level-j segment is below 10^(19 * 2^j) < 2^(64 * 2^j), so it fits in
// 2^j limbs and every level is one array of the same 2^J limbs.  The first
// levels (segments of up to 128 limbs, 2432 digits) are built in one kernel
// by Horner's rule per segment; each later level is one batch of equal-size
// products (the engine's batch plans) and one segmented carry add of the low
// halves.
#include <cuda_runtime.h>

#include <cstdint>

#include "engine.h"

namespace bgpu {
namespace {

constexpr uint64_t kTen19 = 10000000000000000000ull;
constexpr uint32_t kLeafLimbs = 128;  // limbs per segment built by Horner's rule
constexpr int kAddThreads = 256;
constexpr int kAddPer = 8;
constexpr uint32_t kAddTile = kAddThreads * kAddPer;

// Segment s (w limbs, w <= kLeafLimbs) from decimal positions
// [19 w s, 19 w (s+1)) counted from the least significant digit of dig[0..D)
// (most significant first, values 0..9), by Horner's rule over its w groups
// of 19 digits.
__global__ void k_dec_leaves(const uint8_t* dig, uint64_t D, uint32_t w, uint64_t nseg, uint64_t* out) {
    const uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    uint64_t v[kLeafLimbs];
    for (uint32_t i = 0; i < w; ++i) v[i] = 0;
    for (int g = (int)w - 1; g >= 0; --g) {
        // the 19 digits of group g, most significant first
        uint64_t chunk = 0;
        const uint64_t p0 = 19 * ((uint64_t)w * s + (uint64_t)g);  // position of its lowest digit
        for (int k = 18; k >= 0; --k) {
            const uint64_t pos = p0 + (uint64_t)k;
            chunk = chunk * 10 + (pos < D ? dig[D - 1 - pos] : 0u);
        }
        // v = v * 10^19 + chunk
        uint64_t carry = chunk;
        for (uint32_t i = 0; i < w; ++i) {
            const uint64_t lo = v[i] * kTen19, hi = __umul64hi(v[i], kTen19);
            const uint64_t t = lo + carry;
            carry = hi + (t < lo ? 1u : 0u);
            v[i] = t;
        }
    }
    for (uint32_t i = 0; i < w; ++i) out[s * w + i] = v[i];
}

__device__ __forceinline__ uint32_t compose(uint32_t lo, uint32_t hi) {
    const uint32_t g = (hi & 1u) | ((hi >> 1) & lo & 1u);
    const uint32_t p = (hi >> 1) & (lo >> 1) & 1u;
    return g | (p << 1);
}

// Exclusive scan of the block's thread carry states (2 = identity).
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
        if (lane < nw) s_warp[lane] = w;
    }
    __syncthreads();
    uint32_t before = __shfl_up_sync(0xffffffffu, inc, 1);
    if (lane == 0) before = 2u;
    if (warp > 0) before = compose(s_warp[warp - 1], before);
    *total = s_warp[nw - 1];
    __syncthreads();  // s_warp is reused by the next tile
    return before;
}

// One block per segment p: out[p*w2 .. p*w2 + w2) += lo[2p*w1 .. 2p*w1 + w1)
// (w2 = 2 w1), the carry resolved tile by tile across the segment.
__global__ void __launch_bounds__(kAddThreads) k_seg_add_low(uint64_t* out, const uint64_t* prev, uint32_t w1) {
    const uint64_t p = blockIdx.x;
    const uint32_t w2 = 2 * w1;
    uint64_t* o = out + p * w2;
    const uint64_t* lo = prev + 2 * p * w1;
    uint32_t cin = 0;
    for (uint32_t t0 = 0; t0 < w2; t0 += kAddTile) {
        const uint32_t j0 = t0 + threadIdx.x * kAddPer;
        uint64_t x[kAddPer], y[kAddPer];
        uint32_t st = 2u;
#pragma unroll
        for (int k = 0; k < kAddPer; ++k) {
            const uint32_t j = j0 + (uint32_t)k;
            x[k] = j < w2 ? o[j] : 0ull;
            y[k] = j < w1 ? lo[j] : 0ull;
            const uint64_t t = x[k] + y[k];
            if (j < w2) st = compose(st, (uint32_t)(t < x[k]) | ((uint32_t)(t == ~0ull) << 1));
        }
        uint32_t total;
        const uint32_t before = block_exclusive(st, &total);
        uint64_t c = (before & 1u) | ((before >> 1) & cin);
#pragma unroll
        for (int k = 0; k < kAddPer; ++k) {
            const uint32_t j = j0 + (uint32_t)k;
            if (j >= w2) break;
            const uint64_t t = x[k] + y[k], r = t + c;
            c = (uint64_t)(t < x[k]) | (uint64_t)(r < t);
            o[j] = r;
        }
        cin = (total & 1u) | ((total >> 1) & cin);
    }
}

}  // namespace

cudaError_t launch_dec_leaves(const uint8_t* dig, uint64_t D, uint32_t w, uint64_t nseg, uint64_t* out,
                              cudaStream_t st) {
    k_dec_leaves<<<(uint32_t)((nseg + 127) / 128), 128, 0, st>>>(dig, D, w, nseg, out);
    return cudaGetLastError();
}

cudaError_t launch_seg_add_low(uint64_t* out, const uint64_t* prev, uint32_t w1, uint64_t nseg,
                               cudaStream_t st) {
    k_seg_add_low<<<(uint32_t)nseg, kAddThreads, 0, st>>>(out, prev, w1);
    return cudaGetLastError();
}

}  // namespace bgpu
