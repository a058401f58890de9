// Shared machinery of the transform passes (NTT and FP64 FFT): radix round
// plans, element groups of a round, shared-memory swizzles, programmatic
// dependent launch helpers.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace bgpu {

// Round split of a length-2^L transform into radix-2^r rounds (r <= MAXR),
// top bits first (DIF order).
template <int L, int MAXR = 4>
struct Plan {
    static constexpr int nr = (L + MAXR - 1) / MAXR;
    __host__ __device__ static constexpr int r(int k) { return L / nr + (k < L % nr ? 1 : 0); }
    __host__ __device__ static constexpr int hi(int k) {
        int h = L - 1;
        for (int i = 0; i < k; ++i) h -= r(i);
        return h;
    }
    __host__ __device__ static constexpr int lo(int k) { return hi(k) - r(k) + 1; }
};

// Shared-memory placement of element i (of column col) in a [2^L][C] tile.
// The XOR swizzles make every round's access pattern bank-conflict free
// (rows: checked for L = 5..15; 8-column tiles: L = 2..11) and are bijective.
// Both are linear over GF(2): sidx(i ^ k, col) = sidx(i, col) ^ soff(k), so a
// group's element addresses are one base address XOR compile-time constants.
template <int C>
__host__ __device__ constexpr uint32_t soff(uint32_t i) {
    if constexpr (C == 1)
        return i ^ (((i >> 3) ^ (i >> 4)) & 31u);
    else
        return (i ^ (((i >> 2) ^ (i >> 4)) & 3u)) * C;
}

template <int C>
__device__ __forceinline__ uint32_t sidx(uint32_t i, int col) {
    return soff<C>(i) | (uint32_t)col;
}

// Group g of round K on a [2^L][C] tile: column and base element index.
template <int L, int C, int K, int MAXR = 4>
struct Group {
    static constexpr int R = Plan<L, MAXR>::r(K), HI = Plan<L, MAXR>::hi(K), LO = Plan<L, MAXR>::lo(K);
    static constexpr int G = (1 << (L - R)) * C;
    int col;
    uint32_t base, base_low, a0;
    __device__ __forceinline__ explicit Group(int g) {
        col = g % C;
        const uint32_t q = (uint32_t)(g / C);
        base_low = q & ((1u << LO) - 1u);
        base = ((q >> LO) << (HI + 1)) | base_low;
        a0 = sidx<C>(base, col);
    }
    __device__ __forceinline__ uint32_t idx(int j) const { return base + ((uint32_t)j << LO); }
    // smem address of element j: base's bits [LO, LO+R) are zero, so
    // idx(j) = base ^ (j << LO) and the swizzle splits linearly.
    __device__ __forceinline__ uint32_t at(int j) const { return a0 ^ soff<C>((uint32_t)j << LO); }
};

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialization may start while its predecessor finishes; pdl_wait() blocks
// until every earlier kernel in the stream has completed and its writes are
// visible (a no-op for an ordinary launch), pdl_trigger() lets the next
// kernel's launch begin.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Opt in to large dynamic shared memory.  The default limit (48 KB) covers
// static plus dynamic memory, so kernels with a few KB of static tables opt in
// a little below it too.
template <class K>
static void allow_smem(K k, size_t bytes) {
    if (bytes > 40 * 1024) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Launch with programmatic stream serialization, so the kernel's launch
// overlaps the tail of the previous kernel in the stream (each kernel waits in
// pdl_wait() before touching memory an earlier kernel wrote).
template <class Arg>
static cudaError_t launch_k(void (*k)(Arg), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                            const Arg& arg) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k, arg);
}

}  // namespace bgpu
