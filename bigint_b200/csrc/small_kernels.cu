// Small-size kernels: schoolbook and Karatsuba products (one CTA per product,
// batched or single), and 28-bit <-> 64-bit repacking.  The product bodies
// and the method notes are in small_bodies.cuh.
#include "small_bodies.cuh"

namespace bgpu {

struct SmallArgs {
    const SchoolDesc* descs;  // device array (batch) or nullptr
    SchoolDesc one;           // the single product when descs == nullptr
};

__device__ __forceinline__ SchoolDesc small_desc(const SmallArgs& a) {
    return a.descs ? a.descs[blockIdx.x] : a.one;
}

__global__ void __launch_bounds__(kSbThreads) k_schoolbook(const SmallArgs args) {
    __shared__ SbSmem S;
    schoolbook_body(small_desc(args), S);
}

__global__ void __launch_bounds__(kKaThreads) k_karatsuba(const SmallArgs args) {
    __shared__ KaSmem S;
    karatsuba_body(small_desc(args), S);
}

// ---- launchers -----------------------------------------------------------------

cudaError_t launch_schoolbook(const uint64_t* a, uint32_t na, const uint64_t* b, uint32_t nb,
                              uint64_t* out, cudaStream_t stream) {
    if (na == 0 || nb == 0 || na + nb > kSchoolbookMaxLimbs) return cudaErrorInvalidValue;
    SmallArgs args{nullptr, SchoolDesc{a, b, out, na, nb}};
    k_schoolbook<<<1, kSbThreads, 0, stream>>>(args);
    return cudaGetLastError();
}

cudaError_t launch_schoolbook_batch(const SchoolDesc* d_descs, uint32_t count, cudaStream_t stream) {
    if (count == 0) return cudaSuccess;
    SmallArgs args{d_descs, SchoolDesc{}};
    k_schoolbook<<<count, kSbThreads, 0, stream>>>(args);
    return cudaGetLastError();
}

cudaError_t launch_karatsuba(const uint64_t* a, uint32_t na, const uint64_t* b, uint32_t nb,
                             uint64_t* out, cudaStream_t stream) {
    if (na == 0 || nb == 0 || na > kKaratsubaMaxLimbs || nb > kKaratsubaMaxLimbs)
        return cudaErrorInvalidValue;
    SmallArgs args{nullptr, SchoolDesc{a, b, out, na, nb}};
    k_karatsuba<<<1, kKaThreads, 0, stream>>>(args);
    return cudaGetLastError();
}

cudaError_t launch_karatsuba_batch(const SchoolDesc* d_descs, uint32_t count, cudaStream_t stream) {
    if (count == 0) return cudaSuccess;
    SmallArgs args{d_descs, SchoolDesc{}};
    k_karatsuba<<<count, kKaThreads, 0, stream>>>(args);
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
