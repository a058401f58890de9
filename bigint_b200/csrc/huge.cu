// Limb accumulation: out[0, L) += add[0, nadd) with full carry propagation.
//
// Used by the pairwise fallback for products beyond the largest transform
// (the three-prime NTT stops at 2^26 points, 2^31 product bits; the reference
// goes on with Schoenhage-Strassen, src/mul/ssa.cpp:383, chosen by _mul above
// its NTT capacity, include/bigint/mul.h:199-205): there every pair of
// operand blocks is one NTT product, added into the result at its limb offset
// by a carry scan over the rest of the result,
//   A * B = sum_{i,j} (A_i * B_j) * 2^(64 S (i + j)).
// (The default form for those sizes, the spectral sums in engine.cu, carries
// each sum into its window of the result and needs no accumulation.)  Also
// used by the decimal conversions (their power tables and level sums).  Three launches per
// accumulation -- per-block (generate, propagate) aggregates, one block
// scanning them, every block applying its carry-in -- with no inter-block
// waits.
#include <cuda_runtime.h>

#include <cstdint>

#include "engine.h"

namespace bgpu {
namespace {

constexpr int kAccThreads = 256;
constexpr int kAccPer = 8;  // consecutive limbs per thread
constexpr uint32_t kAccBlock = kAccThreads * kAccPer;
constexpr int kAccScanThreads = 1024;

// Carry state of a limb run: bit 0 generate, bit 1 propagate; compose(lo, hi)
// is lo followed by hi.
__device__ __forceinline__ uint32_t compose(uint32_t lo, uint32_t hi) {
    const uint32_t g = (hi & 1u) | ((hi >> 1) & lo & 1u);
    const uint32_t p = (hi >> 1) & (lo >> 1) & 1u;
    return g | (p << 1);
}

struct AccArgs {
    uint64_t* out;       // L limbs, += add
    const uint64_t* add;  // nadd <= L limbs
    uint64_t L;
    uint64_t nadd;
};

__device__ __forceinline__ uint32_t limb_state(uint64_t x, uint64_t y) {
    const uint64_t t = x + y;
    return (uint32_t)(t < x) | ((uint32_t)(t == ~0ull) << 1);
}

__device__ __forceinline__ uint32_t thread_state(const AccArgs& a, uint64_t j0) {
    uint32_t s = 2u;
#pragma unroll
    for (int k = 0; k < kAccPer; ++k) {
        const uint64_t j = j0 + (uint64_t)k;
        if (j < a.L) s = compose(s, limb_state(a.out[j], j < a.nadd ? a.add[j] : 0ull));
    }
    return s;
}

// Exclusive scan of the block's thread states (2 = identity for thread 0);
// *total gets the block's state.
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
    if (total) *total = s_warp[nw - 1];
    return before;
}

__global__ void __launch_bounds__(kAccThreads) k_acc_aggregate(const AccArgs a, uint32_t* agg) {
    const uint64_t j0 = (uint64_t)blockIdx.x * kAccBlock + threadIdx.x * kAccPer;
    uint32_t total;
    block_exclusive(thread_state(a, j0), &total);
    if (threadIdx.x == 0) agg[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kAccScanThreads) k_acc_scan(const uint32_t* agg, uint32_t nblk, uint32_t* cin) {
    const uint32_t per = (nblk + kAccScanThreads - 1) / kAccScanThreads;
    const uint32_t b0 = threadIdx.x * per;
    uint32_t s = 2u;
    for (uint32_t k = 0; k < per; ++k)
        if (b0 + k < nblk) s = compose(s, agg[b0 + k]);
    uint32_t before = block_exclusive(s, nullptr);
    for (uint32_t k = 0; k < per; ++k) {
        if (b0 + k >= nblk) break;
        cin[b0 + k] = before & 1u;
        before = compose(before, agg[b0 + k]);
    }
}

__global__ void __launch_bounds__(kAccThreads) k_acc_apply(const AccArgs a, const uint32_t* cin) {
    const uint64_t j0 = (uint64_t)blockIdx.x * kAccBlock + threadIdx.x * kAccPer;
    const uint32_t before = block_exclusive(thread_state(a, j0), nullptr);
    uint64_t c = (before & 1u) | ((before >> 1) & cin[blockIdx.x]);
#pragma unroll
    for (int k = 0; k < kAccPer; ++k) {
        const uint64_t j = j0 + (uint64_t)k;
        if (j >= a.L) break;
        const uint64_t x = a.out[j], y = j < a.nadd ? a.add[j] : 0ull;
        const uint64_t t = x + y;
        const uint64_t r = t + c;
        c = (uint64_t)(t < x) | (uint64_t)(r < t);
        a.out[j] = r;
    }
}

}  // namespace

uint32_t accumulate_blocks(uint64_t L) { return (uint32_t)((L + kAccBlock - 1) / kAccBlock); }

cudaError_t launch_accumulate(uint64_t* out, uint64_t L, const uint64_t* add, uint64_t nadd, uint32_t* agg,
                              uint32_t* cin, cudaStream_t st) {
    const AccArgs a{out, add, L, nadd};
    const uint32_t nblk = accumulate_blocks(L);
    k_acc_aggregate<<<nblk, kAccThreads, 0, st>>>(a, agg);
    k_acc_scan<<<1, kAccScanThreads, 0, st>>>(agg, nblk, cin);
    k_acc_apply<<<nblk, kAccThreads, 0, st>>>(a, cin);
    return cudaGetLastError();
}

}  // namespace bgpu
