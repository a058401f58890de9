// Decimal text to binary on the device (the reference's BigInt(const
// std::string&) with convert_from_dec_string, src/bigint.cpp:25-124).
//
// The digit string is cut into leaves of 19 digits (one u64 each) from its
// least significant end, and leaves are paired level by level:
//   segment_{j+1}[p] = segment_j[2p+1] * 10^(19 * 2^j) + segment_j[2p].
// A level-j segment is below 10^(19 * 2^j) < 2^(64 * 2^j), so it fits in
// 2^j limbs and every level is one array of the same 2^J limbs.  The first
// levels (segments of up to kParseLeafLimbs = 32 limbs, 608 digits) are built in one kernel
// by Horner's rule per segment; each later level is one batch of equal-size
// products (the engine's batch plans) and one segmented carry add of the low
// halves.
#include <cuda_runtime.h>

#include <cstdint>

#include "engine.h"

namespace bgpu {
namespace {

constexpr uint64_t kTen19 = 10000000000000000000ull;
constexpr int kAddThreads = 256;
constexpr int kAddPer = 8;
constexpr uint32_t kAddTile = kAddThreads * kAddPer;
constexpr int kWideAddThreads = 1024;
constexpr uint32_t kWideDivstepLimbs = 4096;  // w at which a level's divide step uses 1024-thread blocks

// Segment s (w limbs, w <= kParseLeafLimbs) from decimal positions
// [19 w s, 19 w (s+1)) counted from the least significant digit of dig[0..D)
// (most significant first, values 0..9), by Horner's rule over its w groups
// of 19 digits.
__global__ void k_dec_leaves(const uint8_t* dig, uint64_t D, uint32_t w, uint64_t nseg, uint64_t* out) {
    const uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    uint64_t v[kParseLeafLimbs];
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

// ---- binary to decimal -------------------------------------------------------
//
// The reverse walk: a level-j segment s < Q^2 (Q = 10^(19 w), w = 2^(j-1)
// limbs) splits into s div Q and s mod Q.  The host has the exact reciprocal
// V = floor(2^(128 w) / Q) and T = s * V and U = (T >> 128 w) * Q as batched
// products; q = T >> 128 w is q_true or q_true - 1 (V exact, s < 2^(128 w)).
// One block per segment then forms r = s - U and, when r >= Q, subtracts Q
// once more and adds 1 to q.

// Block-wide sum or difference of two limb runs with the carry (or borrow)
// carried across tiles of T * kAddPer limbs (T = the block's threads); out
// may alias x.  Returns the carry out.
template <int T>
__device__ uint32_t block_addsub(uint64_t* out, const uint64_t* x, uint32_t nx, const uint64_t* y, uint32_t ny,
                                 uint32_t n, bool sub, uint32_t cin) {
    for (uint32_t t0 = 0; t0 < n; t0 += (uint32_t)T * kAddPer) {
        const uint32_t j0 = t0 + threadIdx.x * kAddPer;
        uint64_t a[kAddPer], b[kAddPer];
        uint32_t st = 2u;
#pragma unroll
        for (int k = 0; k < kAddPer; ++k) {
            const uint32_t j = j0 + (uint32_t)k;
            a[k] = j < nx ? x[j] : 0ull;
            b[k] = j < ny ? y[j] : 0ull;
            uint32_t g, pr;
            if (sub) {
                g = a[k] < b[k];
                pr = a[k] == b[k];
            } else {
                const uint64_t t = a[k] + b[k];
                g = t < a[k];
                pr = t == ~0ull;
            }
            if (j < n) st = compose(st, g | (pr << 1));
        }
        uint32_t total;
        const uint32_t before = block_exclusive(st, &total);
        uint64_t c = (before & 1u) | ((before >> 1) & cin);
#pragma unroll
        for (int k = 0; k < kAddPer; ++k) {
            const uint32_t j = j0 + (uint32_t)k;
            if (j >= n) break;
            if (sub) {
                const uint64_t t = a[k] - b[k], r = t - c;
                c = (uint64_t)(a[k] < b[k]) | (uint64_t)(t < c);
                out[j] = r;
            } else {
                const uint64_t t = a[k] + b[k], r = t + c;
                c = (uint64_t)(t < a[k]) | (uint64_t)(r < t);
                out[j] = r;
            }
        }
        cin = (total & 1u) | ((total >> 1) & cin);
        __syncthreads();  // the next tile reads what this one wrote only through its own indices
    }
    return cin;
}

// 1 when x (nx limbs) >= y (ny limbs), block-wide.
__device__ bool block_geq(const uint64_t* x, uint32_t nx, const uint64_t* y, uint32_t ny) {
    __shared__ unsigned long long s_key;
    if (threadIdx.x == 0) s_key = 0;
    __syncthreads();
    const uint32_t n = nx > ny ? nx : ny;
    unsigned long long best = 0;
    for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
        const uint64_t a = j < nx ? x[j] : 0ull, b = j < ny ? y[j] : 0ull;
        if (a != b) best = ((unsigned long long)(j + 1) << 1) | (a > b ? 1u : 0u);
    }
    if (best) atomicMax(&s_key, best);
    __syncthreads();
    const unsigned long long key = s_key;
    __syncthreads();
    return key == 0 || (key & 1u);
}

// Segment p of the level above (2w limbs at cur + 2 w p) with U_p = q * Q
// (2w limbs at u + 2 w p) and q (w limbs at t + (2w + m) p + 2w) written as
// the two halves of the level below: next[2 w p ..] = r, next[2 w p + w ..] = q.
template <int T>
__global__ void __launch_bounds__(T) k_seg_divstep(const uint64_t* cur, uint64_t* u, uint64_t* t, uint32_t tstride,
                                                   const uint64_t* q_pow, uint32_t w, uint64_t* next) {
    const uint64_t p = blockIdx.x;
    const uint64_t* s = cur + 2 * (uint64_t)w * p;
    uint64_t* r = u + 2 * (uint64_t)w * p;
    uint64_t* q = t + (uint64_t)tstride * p + 2 * w;
    block_addsub<T>(r, s, 2 * w, r, 2 * w, 2 * w, true, 0);  // r = s - q Q, in place of U
    __syncthreads();
    if (block_geq(r, 2 * w, q_pow, w)) {  // q was one short
        block_addsub<T>(r, r, 2 * w, q_pow, w, 2 * w, true, 0);
        __syncthreads();
        block_addsub<T>(q, q, w, nullptr, 0, w, false, 1);
        __syncthreads();
    }
    uint64_t* lo = next + 2 * (uint64_t)w * p;
    for (uint32_t j = threadIdx.x; j < w; j += blockDim.x) {
        lo[j] = r[j];
        lo[w + j] = q[j];
    }
}

// Decimal text of segment p (w limbs, value < 10^(19 w)): 19 w characters,
// most significant first, at out + 19 w (nseg - 1 - p); by repeated division
// of its 32-bit halves by 10^9.
__global__ void k_dec_print_leaves(const uint64_t* in, uint32_t w, uint64_t nseg, char* out) {
    const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nseg) return;
    uint32_t x[2 * kPrintLeafLimbs];
    const uint32_t nw = 2 * w;
    for (uint32_t i = 0; i < w; ++i) {
        const uint64_t v = in[p * w + i];
        x[2 * i] = (uint32_t)v;
        x[2 * i + 1] = (uint32_t)(v >> 32);
    }
    const uint32_t nchar = 19 * w;
    char* o = out + (uint64_t)nchar * (nseg - 1 - p);
    uint32_t top = nw;  // words above top are zero
    for (uint32_t done = 0; done < nchar; done += 9) {
        while (top > 0 && x[top - 1] == 0) --top;
        uint64_t rem = 0;
        for (uint32_t i = top; i-- > 0;) {
            const uint64_t cur = (rem << 32) | x[i];
            x[i] = (uint32_t)(cur / 1000000000u);
            rem = cur % 1000000000u;
        }
        for (uint32_t k = 0; k < 9 && done + k < nchar; ++k) {
            o[nchar - 1 - (done + k)] = (char)('0' + rem % 10);
            rem /= 10;
        }
    }
}

// r[i] = ~x[i] for i < el, r[el] = 0 (then r + 1 = 2^(64 el) - x for 0 < x < 2^(64 el)).
__global__ void k_not_limbs(const uint64_t* x, uint32_t el, uint64_t* r) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= el; i += gridDim.x * blockDim.x)
        r[i] = i < el ? ~x[i] : 0ull;
}

// One block: when r (nr limbs) >= q (nq limbs), r -= q and v += 1 (nv limbs);
// *flag = 1 if it did.
__global__ void __launch_bounds__(kAddThreads) k_fix_step(uint64_t* r, uint32_t nr, const uint64_t* q, uint32_t nq,
                                                          uint64_t* v, uint32_t nv, uint32_t* flag) {
    const bool ge = block_geq(r, nr, q, nq);
    if (ge) {
        block_addsub<kAddThreads>(r, r, nr, q, nq, nr, true, 0);
        __syncthreads();
        block_addsub<kAddThreads>(v, v, nv, nullptr, 0, nv, false, 1);
    }
    if (threadIdx.x == 0) *flag = ge ? 1u : 0u;
}

}  // namespace

cudaError_t launch_not_limbs(const uint64_t* x, uint32_t el, uint64_t* r, cudaStream_t st) {
    k_not_limbs<<<(el + 256) / 256 < 1184 ? (el + 256) / 256 : 1184, 256, 0, st>>>(x, el, r);
    return cudaGetLastError();
}

cudaError_t launch_fix_step(uint64_t* r, uint32_t nr, const uint64_t* q, uint32_t nq, uint64_t* v, uint32_t nv,
                            uint32_t* flag, cudaStream_t st) {
    k_fix_step<<<1, kAddThreads, 0, st>>>(r, nr, q, nq, v, nv, flag);
    return cudaGetLastError();
}

cudaError_t launch_seg_divstep(const uint64_t* cur, uint64_t* u, uint64_t* t, uint32_t tstride, const uint64_t* q_pow,
                               uint32_t w, uint64_t nseg, uint64_t* next, cudaStream_t st) {
    // long segments (the top levels: few of them, one block each) walk their
    // limbs in 4x wider tiles
    if (w >= kWideDivstepLimbs)
        k_seg_divstep<kWideAddThreads><<<(uint32_t)nseg, kWideAddThreads, 0, st>>>(cur, u, t, tstride, q_pow, w, next);
    else
        k_seg_divstep<kAddThreads><<<(uint32_t)nseg, kAddThreads, 0, st>>>(cur, u, t, tstride, q_pow, w, next);
    return cudaGetLastError();
}

cudaError_t launch_dec_print_leaves(const uint64_t* in, uint32_t w, uint64_t nseg, char* out, cudaStream_t st) {
    if (w > kPrintLeafLimbs) return cudaErrorInvalidValue;
    k_dec_print_leaves<<<(uint32_t)((nseg + 63) / 64), 64, 0, st>>>(in, w, nseg, out);
    return cudaGetLastError();
}

cudaError_t launch_dec_leaves(const uint8_t* dig, uint64_t D, uint32_t w, uint64_t nseg, uint64_t* out,
                              cudaStream_t st) {
    if (w > kParseLeafLimbs) return cudaErrorInvalidValue;
    k_dec_leaves<<<(uint32_t)((nseg + 127) / 128), 128, 0, st>>>(dig, D, w, nseg, out);
    return cudaGetLastError();
}

cudaError_t launch_seg_add_low(uint64_t* out, const uint64_t* prev, uint32_t w1, uint64_t nseg,
                               cudaStream_t st) {
    k_seg_add_low<<<(uint32_t)nseg, kAddThreads, 0, st>>>(out, prev, w1);
    return cudaGetLastError();
}

}  // namespace bgpu
