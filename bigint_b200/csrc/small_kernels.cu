// Small-size kernels: schoolbook product and 28-bit <-> 64-bit repacking.
//
// Schoolbook follows the reference's brute::mul (include/bigint/mul.h:82-102)
// in what it computes; on the GPU each thread owns one output column
// (sum of a_i * b_{k-i} as a 192-bit accumulator) and the column sums are
// folded into limbs by a short carry pass.
#include "engine.h"

namespace bgpu {

constexpr int kSchoolThreads = 256;

__global__ void __launch_bounds__(kSchoolThreads)
    k_schoolbook(const uint64_t* __restrict__ a, uint32_t na, const uint64_t* __restrict__ b,
                 uint32_t nb, uint64_t* __restrict__ out) {
    __shared__ uint64_t sa[kSchoolbookMaxLimbs], sb[kSchoolbookMaxLimbs];
    __shared__ uint64_t c0[kSchoolbookMaxLimbs], c1[kSchoolbookMaxLimbs], c2[kSchoolbookMaxLimbs];
    for (uint32_t i = threadIdx.x; i < na; i += kSchoolThreads) sa[i] = a[i];
    for (uint32_t i = threadIdx.x; i < nb; i += kSchoolThreads) sb[i] = b[i];
    __syncthreads();
    const uint32_t ncol = na + nb;
    for (uint32_t k = threadIdx.x; k < ncol; k += kSchoolThreads) {
        uint64_t x0 = 0, x1 = 0, x2 = 0;
        if (k + 1 < ncol) {
            const uint32_t i0 = k + 1 > nb ? k + 1 - nb : 0;
            const uint32_t i1 = k < na - 1 ? k : na - 1;
            for (uint32_t i = i0; i <= i1; ++i) {
                const uint64_t u = sa[i], v = sb[k - i];
                const uint64_t lo = u * v, hi = __umul64hi(u, v);
                x0 += lo;
                const uint64_t c = x0 < lo;
                const uint64_t t = x1 + hi;
                x2 += (t < x1);
                x1 = t + c;
                x2 += (x1 < c);
            }
        }
        c0[k] = x0, c1[k] = x1, c2[k] = x2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned __int128 carry = 0;
        for (uint32_t k = 0; k < ncol; ++k) {
            unsigned __int128 s = carry + c0[k];
            if (k >= 1) s += c1[k - 1];
            if (k >= 2) s += c2[k - 2];
            out[k] = (uint64_t)s;
            carry = s >> 64;
        }
    }
}

cudaError_t launch_schoolbook(const uint64_t* a, uint32_t na, const uint64_t* b, uint32_t nb,
                              uint64_t* out, cudaStream_t stream) {
    if (na == 0 || nb == 0 || na + nb > kSchoolbookMaxLimbs) return cudaErrorInvalidValue;
    k_schoolbook<<<1, kSchoolThreads, 0, stream>>>(a, na, b, nb, out);
    return cudaGetLastError();
}

// limbs[w] = bits [64w, 64w+64) of sum d[i] 2^(28 i).
__global__ void k_digits28_to_limbs(const uint32_t* __restrict__ d, uint32_t nd,
                                    uint64_t* __restrict__ limbs, uint32_t nlimbs) {
    const uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nlimbs) return;
    const uint64_t bit0 = (uint64_t)w * 64;
    uint32_t i = (uint32_t)(bit0 / 28);
    uint64_t v = 0;
    for (; i < nd; ++i) {
        const int64_t off = (int64_t)i * 28 - (int64_t)bit0;  // digit start relative to limb
        if (off >= 64) break;
        const uint64_t dv = d[i];
        v |= off >= 0 ? (dv << off) : (dv >> (-off));
    }
    limbs[w] = v;
}

// d[k] = bits [28k, 28k+28) of the limb array.
__global__ void k_limbs_to_digits28(const uint64_t* __restrict__ limbs, uint32_t nlimbs,
                                    uint32_t* __restrict__ d, uint32_t nd) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nd) return;
    const uint64_t bit = (uint64_t)k * 28;
    const uint32_t w = (uint32_t)(bit >> 6), sh = (uint32_t)(bit & 63);
    uint64_t v = w < nlimbs ? limbs[w] >> sh : 0;
    if (sh > 36 && w + 1 < nlimbs) v |= limbs[w + 1] << (64 - sh);
    d[k] = (uint32_t)v & ((1u << 28) - 1u);
}

cudaError_t launch_digits28_to_limbs(const uint32_t* d, uint32_t nd, uint64_t* limbs,
                                     uint32_t nlimbs, cudaStream_t stream) {
    k_digits28_to_limbs<<<(nlimbs + 255) / 256, 256, 0, stream>>>(d, nd, limbs, nlimbs);
    return cudaGetLastError();
}

cudaError_t launch_limbs_to_digits28(const uint64_t* limbs, uint32_t nlimbs, uint32_t* d,
                                     uint32_t nd, cudaStream_t stream) {
    k_limbs_to_digits28<<<(nd + 255) / 256, 256, 0, stream>>>(limbs, nlimbs, d, nd);
    return cudaGetLastError();
}

}  // namespace bgpu
