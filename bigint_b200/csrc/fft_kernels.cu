// FP64 complex-FFT product pipeline (the reference's fft::mul form,
// src/mul/fft.cpp:281-384), built on the same two-pass layout as the NTT.
//
// Operands are split into b-bit points; A goes into the real part and B into
// the imaginary part of one complex vector (fft.cpp:330-338), so a single
// forward transform covers both.  After the pointwise square,
// (A + iB)^2 = A^2 - B^2 + 2i(A*B), the inverse transform's imaginary part
// divided by 2 is the convolution A*B (fft.cpp:342-364).  Five launches:
//   k_fft_fwd_cols  points -> length-N2 DIF per column tile, twiddle
//   k_fft_mid_rows  length-N1 DIF per row, square, DIT back, twiddle
//   k_fft_inv_cols  length-N2 DIT, 1/N, coefficient = round(Im/2), and the
//                   block maximum of |Im/2 - round(Im/2)| into a device word
//   k_fft_chunks    coefficients at bit offsets b*k -> 256-bit chunk sums
//   k_carry         (shared with the NTT) carry scan and output
// Twiddles are host-computed FP64 tables (long-double sin/cos, rounded), so
// each is within one rounding of the exact root; no recurrences are used
// (the reference chains seed*step, fft.cpp:78-102).
#include <cuda/atomic>

#include "engine.h"
#include "pass_common.cuh"

namespace bgpu {

// Columns per column tile: 4 (64 B per row segment) up to 2^11 rows; 2 and 1
// for the 2^12- and 2^13-row columns of the largest transforms, so a tile
// stays at 128 KB of shared memory.
__host__ __device__ constexpr int fft_cols(int l2) { return l2 <= 11 ? 4 : (l2 == 12 ? 2 : 1); }
constexpr int kFftMaxR = 3;  // radix-8 rounds (double2 data: 16 values per thread)

__constant__ FftConsts c_fft;

cudaError_t upload_fft_consts(const FftConsts& c) { return cudaMemcpyToSymbol(c_fft, &c, sizeof(c)); }

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csubd(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 w) {
    return make_double2(fma(a.x, w.x, -a.y * w.y), fma(a.x, w.y, a.y * w.x));
}

// Shared-memory placement for 16-byte elements.  Column tiles of 4 columns
// put row i at slots 4*swz(i) .. 4*swz(i)+3, swz(i) = i with bit 0 flipped by
// the parity of the higher bits: the two rows an 8-lane phase touches always
// differ by one power of two, so they land in opposite halves of a 128-byte
// window (conflict free).  Rows use an XOR-linear, bijective swizzle that
// keeps 8-lane phases conflict free.  Both are linear over GF(2).
__host__ __device__ constexpr uint32_t parity32(uint32_t v) {
    v ^= v >> 16;
    v ^= v >> 8;
    v ^= v >> 4;
    v ^= v >> 2;
    v ^= v >> 1;
    return v & 1u;
}

template <int C>
__host__ __device__ constexpr uint32_t fsoff(uint32_t i) {
    if constexpr (C == 1)
        return i ^ (((i >> 2) ^ (i >> 5)) & 7u);
    else
        return (i ^ parity32(i >> 1)) * C;
}

template <int L, int C, int K>
struct FGroup {
    using P = Plan<L, kFftMaxR>;
    static constexpr int R = P::r(K), HI = P::hi(K), LO = P::lo(K);
    static constexpr int G = (1 << (L - R)) * C;
    int col;
    uint32_t base, base_low, a0;
    __device__ __forceinline__ explicit FGroup(int g) {
        col = g % C;
        const uint32_t q = (uint32_t)(g / C);
        base_low = q & ((1u << LO) - 1u);
        base = ((q >> LO) << (HI + 1)) | base_low;
        a0 = fsoff<C>(base) | (uint32_t)col;
    }
    __device__ __forceinline__ uint32_t idx(int j) const { return base + ((uint32_t)j << LO); }
    __device__ __forceinline__ uint32_t at(int j) const { return a0 ^ fsoff<C>((uint32_t)j << LO); }
};

template <int R, int HI, int LO>
__device__ __forceinline__ void fdif(double2 (&x)[1 << R], uint32_t base_low, const double2* tw) {
    const double2* twb = tw + base_low;
#pragma unroll
    for (int t = 0; t < R; ++t) {
        const uint32_t h = 1u << (HI - t);
        const int dist = 1 << (R - 1 - t);
#pragma unroll
        for (int j = 0; j < (1 << R); ++j) {
            if (j & dist) continue;
            const double2 a = x[j], b = x[j + dist];
            x[j] = cadd(a, b);
            if (LO == 0 && (j & (dist - 1)) == 0)
                x[j + dist] = csubd(a, b);
            else
                x[j + dist] = cmul(csubd(a, b), __ldg(twb + h + ((uint32_t)(j & (dist - 1)) << LO)));
        }
    }
}

template <int R, int HI, int LO>
__device__ __forceinline__ void fdit(double2 (&x)[1 << R], uint32_t base_low, const double2* tw) {
    const double2* twb = tw + base_low;
#pragma unroll
    for (int t = R - 1; t >= 0; --t) {
        const uint32_t h = 1u << (HI - t);
        const int dist = 1 << (R - 1 - t);
#pragma unroll
        for (int j = 0; j < (1 << R); ++j) {
            if (j & dist) continue;
            double2 b = x[j + dist];
            if (!(LO == 0 && (j & (dist - 1)) == 0))
                b = cmul(b, __ldg(twb + h + ((uint32_t)(j & (dist - 1)) << LO)));
            const double2 a = x[j];
            x[j] = cadd(a, b);
            x[j + dist] = csubd(a, b);
        }
    }
}

template <int L, int C, int T, int K, bool INV>
__device__ __forceinline__ void fround(double2* sm, const double2* tw, int tid) {
    using Gr = FGroup<L, C, K>;
    constexpr int R = Gr::R;
#pragma unroll 1
    for (int g = tid; g < Gr::G; g += T) {
        const Gr gr(g);
        double2 x[1 << R];
#pragma unroll
        for (int j = 0; j < (1 << R); ++j) x[j] = sm[gr.at(j)];
        if constexpr (INV)
            fdit<R, Gr::HI, Gr::LO>(x, gr.base_low, tw);
        else
            fdif<R, Gr::HI, Gr::LO>(x, gr.base_low, tw);
#pragma unroll
        for (int j = 0; j < (1 << R); ++j) sm[gr.at(j)] = x[j];
    }
}

template <int L, int C, int T, int K, int KEND>
__device__ __forceinline__ void fdif_rounds(double2* sm, const double2* tw) {
    if constexpr (K <= KEND) {
        fround<L, C, T, K, false>(sm, tw, threadIdx.x);
        __syncthreads();
        fdif_rounds<L, C, T, K + 1, KEND>(sm, tw);
    }
}

template <int L, int C, int T, int K, int KEND>
__device__ __forceinline__ void fdit_rounds(double2* sm, const double2* tw) {
    if constexpr (K >= KEND) {
        fround<L, C, T, K, true>(sm, tw, threadIdx.x);
        __syncthreads();
        fdit_rounds<L, C, T, K - 1, KEND>(sm, tw);
    }
}

// omega_N^(+-e) from the two split tables (one complex multiply).
__device__ __forceinline__ double2 ftwiddle(int dir, uint32_t e, int log_n) {
    const uint32_t em = e << (c_fft.log_max - log_n);
    const double2 hi = __ldg(c_fft.th[dir] + (em >> c_fft.split));
    const double2 lo = __ldg(c_fft.tl[dir] + (em & ((1u << c_fft.split) - 1u)));
    return cmul(hi, lo);
}

// b-bit point k of a limb array of n limbs (0 beyond it).
__device__ __forceinline__ double point(const uint64_t* x, uint32_t n, uint64_t k, int b) {
    const uint64_t bit = k * (uint64_t)b;
    const uint64_t w = bit >> 6;
    if (w >= n) return 0.0;
    const uint32_t s = (uint32_t)(bit & 63);
    uint64_t v = __ldg(x + w) >> s;
    if (s + b > 64 && w + 1 < n) v |= __ldg(x + w + 1) << (64 - s);
    return (double)(v & ((1ull << b) - 1ull));
}

struct FftFwdArgs {
    const uint64_t* a;
    const uint64_t* b;  // == a when squaring
    uint32_t na, nb;
    int bits;
    double2* y;
    int log_n, log_n1;
};

template <int L2, int T>
__global__ void __launch_bounds__(T) k_fft_fwd_cols(const FftFwdArgs a) {
    constexpr int kFftCols = fft_cols(L2);
    extern __shared__ __align__(16) double2 fsm[];  // [2^L2][kFftCols]
    using P2 = Plan<L2, kFftMaxR>;
    constexpr int NR = P2::nr;
    const double2* tw = c_fft.stage[0];
    const uint32_t n1_len = 1u << a.log_n1, c0 = blockIdx.x * kFftCols;
    const uint32_t nmask = (1u << a.log_n) - 1u;
    pdl_wait();
    pdl_trigger();
    {
        using Gr = FGroup<L2, kFftCols, 0>;
        constexpr int R = Gr::R;
#pragma unroll 1
        for (int g = threadIdx.x; g < Gr::G; g += T) {
            const Gr gr(g);
            double2 x[1 << R];
#pragma unroll
            for (int j = 0; j < (1 << R); ++j) {
                const uint64_t n = c0 + gr.col + (uint64_t)n1_len * gr.idx(j);
                x[j] = make_double2(point(a.a, a.na, n, a.bits), point(a.b, a.nb, n, a.bits));
            }
            fdif<R, Gr::HI, Gr::LO>(x, gr.base_low, tw);
            if constexpr (NR == 1) {
#pragma unroll
                for (int j = 0; j < (1 << R); ++j) {
                    const uint32_t slot = gr.idx(j), n1 = c0 + gr.col;
                    const double2 w = ftwiddle(0, (n1 * (__brev(slot) >> (32 - L2))) & nmask, a.log_n);
                    a.y[(size_t)slot * n1_len + n1] = cmul(x[j], w);
                }
            } else {
#pragma unroll
                for (int j = 0; j < (1 << R); ++j) fsm[gr.at(j)] = x[j];
            }
        }
    }
    if constexpr (NR > 1) {
        __syncthreads();
        fdif_rounds<L2, kFftCols, T, 1, NR - 2>(fsm, tw);
        using Gr = FGroup<L2, kFftCols, NR - 1>;
        constexpr int R = Gr::R;
#pragma unroll 1
        for (int g = threadIdx.x; g < Gr::G; g += T) {
            const Gr gr(g);
            double2 x[1 << R];
#pragma unroll
            for (int j = 0; j < (1 << R); ++j) x[j] = fsm[gr.at(j)];
            fdif<R, Gr::HI, Gr::LO>(x, gr.base_low, tw);
            const uint32_t n1 = c0 + gr.col;
#pragma unroll
            for (int j = 0; j < (1 << R); ++j) {
                const uint32_t slot = gr.idx(j);
                const double2 w = ftwiddle(0, (n1 * (__brev(slot) >> (32 - L2))) & nmask, a.log_n);
                a.y[(size_t)slot * n1_len + n1] = cmul(x[j], w);
            }
        }
    }
}

struct FftMidArgs {
    double2* y;
    int log_n, log_n2;
};

template <int L1, int T>
__global__ void __launch_bounds__(T) k_fft_mid_rows(const FftMidArgs a) {
    extern __shared__ __align__(16) double2 fsm[];  // [2^L1]
    using P1 = Plan<L1, kFftMaxR>;
    constexpr int NR = P1::nr;
    const double2* twf = c_fft.stage[0];
    const double2* twi = c_fft.stage[1];
    const uint32_t slot = blockIdx.x;
    const uint32_t nmask = (1u << a.log_n) - 1u;
    double2* row = a.y + (size_t)slot * (1u << L1);
    const uint32_t k2 = a.log_n2 ? (__brev(slot) >> (32 - a.log_n2)) : 0u;
    pdl_wait();
    pdl_trigger();
    // Round 0 from global.
    {
        using Gr = FGroup<L1, 1, 0>;
        constexpr int R = Gr::R;
#pragma unroll 1
        for (int g = threadIdx.x; g < Gr::G; g += T) {
            const Gr gr(g);
            double2 x[1 << R];
#pragma unroll
            for (int j = 0; j < (1 << R); ++j) x[j] = row[gr.idx(j)];
            fdif<R, Gr::HI, Gr::LO>(x, gr.base_low, twf);
            if constexpr (NR == 1) {
#pragma unroll
                for (int j = 0; j < (1 << R); ++j)
                    x[j] = make_double2((x[j].x + x[j].y) * (x[j].x - x[j].y), 2.0 * x[j].x * x[j].y);
                fdit<R, Gr::HI, Gr::LO>(x, gr.base_low, twi);
#pragma unroll
                for (int j = 0; j < (1 << R); ++j)
                    row[gr.idx(j)] = cmul(x[j], ftwiddle(1, (gr.idx(j) * k2) & nmask, a.log_n));
            } else {
#pragma unroll
                for (int j = 0; j < (1 << R); ++j) fsm[gr.at(j)] = x[j];
            }
        }
    }
    if constexpr (NR > 1) {
        __syncthreads();
        fdif_rounds<L1, 1, T, 1, NR - 2>(fsm, twf);
        // Last DIF round, pointwise square, first DIT round.
        {
            using Gr = FGroup<L1, 1, NR - 1>;
            constexpr int R = Gr::R;
#pragma unroll 1
            for (int g = threadIdx.x; g < Gr::G; g += T) {
                const Gr gr(g);
                double2 x[1 << R];
#pragma unroll
                for (int j = 0; j < (1 << R); ++j) x[j] = fsm[gr.at(j)];
                fdif<R, Gr::HI, Gr::LO>(x, gr.base_low, twf);
#pragma unroll
                for (int j = 0; j < (1 << R); ++j)
                    x[j] = make_double2((x[j].x + x[j].y) * (x[j].x - x[j].y), 2.0 * x[j].x * x[j].y);
                fdit<R, Gr::HI, Gr::LO>(x, gr.base_low, twi);
#pragma unroll
                for (int j = 0; j < (1 << R); ++j) fsm[gr.at(j)] = x[j];
            }
        }
        __syncthreads();
        fdit_rounds<L1, 1, T, NR - 2, 1>(fsm, twi);
        using Gr = FGroup<L1, 1, 0>;
        constexpr int R = Gr::R;
#pragma unroll 1
        for (int g = threadIdx.x; g < Gr::G; g += T) {
            const Gr gr(g);
            double2 x[1 << R];
#pragma unroll
            for (int j = 0; j < (1 << R); ++j) x[j] = fsm[gr.at(j)];
            fdit<R, Gr::HI, Gr::LO>(x, gr.base_low, twi);
#pragma unroll
            for (int j = 0; j < (1 << R); ++j)
                row[gr.idx(j)] = cmul(x[j], ftwiddle(1, (gr.idx(j) * k2) & nmask, a.log_n));
        }
    }
}

// Distance of a coefficient estimate to the nearest integer.  An estimate at
// or above 2^50 (where consecutive doubles are 1/4 apart) or clearly below
// zero (coefficients are non-negative) cannot be certified and counts as 1.
__device__ __forceinline__ double round_err(double v, double r) {
    if (v >= 0x1p50 || v < -0.25) return 1.0;
    return fabs(v - r);
}

struct FftInvArgs {
    const double2* z;
    uint64_t* coef;              // N coefficients
    unsigned long long* maxerr;  // bit pattern of the largest |x - round(x)| (x >= 0)
    int log_n, log_n1;
};

template <int L2, int T>
__global__ void __launch_bounds__(T) k_fft_inv_cols(const FftInvArgs a) {
    constexpr int kFftCols = fft_cols(L2);
    extern __shared__ __align__(16) double2 fsm[];
    __shared__ double s_err[T / 32];
    using P2 = Plan<L2, kFftMaxR>;
    constexpr int NR = P2::nr;
    const double2* twi = c_fft.stage[1];
    const uint32_t n1_len = 1u << a.log_n1, c0 = blockIdx.x * kFftCols;
    const double half_inv_n = 0.5 / (double)(1u << a.log_n);  // exact power of two
    double err = 0.0;
    pdl_wait();
    pdl_trigger();
    {
        using Gr = FGroup<L2, kFftCols, NR - 1>;
        constexpr int R = Gr::R;
#pragma unroll 1
        for (int g = threadIdx.x; g < Gr::G; g += T) {
            const Gr gr(g);
            double2 x[1 << R];
#pragma unroll
            for (int j = 0; j < (1 << R); ++j) x[j] = a.z[(size_t)gr.idx(j) * n1_len + c0 + gr.col];
            fdit<R, Gr::HI, Gr::LO>(x, gr.base_low, twi);
            if constexpr (NR == 1) {
#pragma unroll
                for (int j = 0; j < (1 << R); ++j) {
                    const double v = x[j].y * half_inv_n;
                    const double r = rint(v);
                    err = fmax(err, round_err(v, r));
                    a.coef[c0 + gr.col + (size_t)n1_len * gr.idx(j)] = r > 0.0 ? (uint64_t)r : 0ull;
                }
            } else {
#pragma unroll
                for (int j = 0; j < (1 << R); ++j) fsm[gr.at(j)] = x[j];
            }
        }
    }
    if constexpr (NR > 1) {
        __syncthreads();
        fdit_rounds<L2, kFftCols, T, NR - 2, 1>(fsm, twi);
        using Gr = FGroup<L2, kFftCols, 0>;
        constexpr int R = Gr::R;
#pragma unroll 1
        for (int g = threadIdx.x; g < Gr::G; g += T) {
            const Gr gr(g);
            double2 x[1 << R];
#pragma unroll
            for (int j = 0; j < (1 << R); ++j) x[j] = fsm[gr.at(j)];
            fdit<R, Gr::HI, Gr::LO>(x, gr.base_low, twi);
#pragma unroll
            for (int j = 0; j < (1 << R); ++j) {
                const double v = x[j].y * half_inv_n;
                const double r = rint(v);
                err = fmax(err, round_err(v, r));
                a.coef[c0 + gr.col + (size_t)n1_len * gr.idx(j)] = r > 0.0 ? (uint64_t)r : 0ull;
            }
        }
    }
    // block maximum of the rounding distance -> one atomic per block
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) err = fmax(err, __shfl_xor_sync(0xffffffffu, err, o));
    if ((threadIdx.x & 31) == 0) s_err[threadIdx.x >> 5] = err;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < T / 32; ++w) m = fmax(m, s_err[w]);
        atomicMax(a.maxerr, (unsigned long long)__double_as_longlong(m));
    }
}

struct FftChunkArgs {
    const uint64_t* coef;
    uint32_t ncoef;  // = N
    int bits;
    uint32_t nchunks;
    uint64_t* chunks;
    uint64_t* spill;
};

// Chunk j = the exact sum of c_k * 2^(b*k - 256 j) over the points starting in
// bits [256 j, 256 j + 256): four limbs plus the overflow word.
__global__ void __launch_bounds__(256) k_fft_chunks(const FftChunkArgs a) {
    pdl_wait();
    pdl_trigger();
    const uint32_t j = blockIdx.x * 256 + threadIdx.x;
    if (j >= a.nchunks) return;
    const uint64_t bit0 = (uint64_t)j * 256;
    const uint64_t k0 = (bit0 + a.bits - 1) / a.bits;
    uint64_t k1 = (bit0 + 256 + a.bits - 1) / a.bits;
    if (k1 > a.ncoef) k1 = a.ncoef;
    uint64_t acc[5] = {0, 0, 0, 0, 0};
    for (uint64_t k = k0; k < k1; ++k) {
        const uint64_t c = __ldg(a.coef + k);
        const uint32_t s = (uint32_t)(k * a.bits - bit0);  // < 256
        const uint32_t w = s >> 6, sh = s & 63;
        const uint64_t lo = c << sh, hi = sh ? (c >> (64 - sh)) : 0ull;
        // add (hi:lo) at limb w, carrying upward (acc[4] never overflows)
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            if ((uint32_t)t == w) {
                uint64_t s0 = acc[t] + lo;
                uint64_t cy = s0 < lo;
                acc[t] = s0;
                uint64_t s1 = acc[t + 1] + hi;
                uint64_t cy1 = s1 < hi;
                s1 += cy;
                cy1 += (s1 < cy);
                acc[t + 1] = s1;
#pragma unroll
                for (int u = t + 2; u < 5; ++u) {
                    const uint64_t v = acc[u] + cy1;
                    cy1 = v < cy1;
                    acc[u] = v;
                }
            }
        }
    }
    ulonglong2* dst = reinterpret_cast<ulonglong2*>(a.chunks + (size_t)j * 4);
    dst[0] = make_ulonglong2(acc[0], acc[1]);
    dst[1] = make_ulonglong2(acc[2], acc[3]);
    a.spill[j] = acc[4];
}

// ---- host launchers ---------------------------------------------------------

FftShape fft_choose_shape(int log_n) {
    FftShape s;
    s.log_n = log_n;
    int l2 = (log_n - 1) / 2;
    if (l2 > 10) l2 = 10;
    if (l2 < 2) l2 = 2;
    if (log_n - l2 > 13) l2 = log_n - 13;  // rows stop at 2^13 points (128 KB of shared memory)
    s.log_n2 = l2;
    s.log_n1 = log_n - l2;
    return s;
}

bool fft_shape_supported(int log_n) {
    if (log_n < 8 || log_n > kFftMaxLogN) return false;
    const FftShape s = fft_choose_shape(log_n);
    return s.log_n1 >= 3 && s.log_n1 <= 13 && s.log_n2 >= 2 && s.log_n2 <= 13;
}

static constexpr int fft_row_threads(int l1) { return l1 >= 11 ? 256 : (l1 >= 8 ? (1 << (l1 - 3)) : 32); }

template <int L2>
static cudaError_t fft_outer(const FftFwdArgs* f, const FftInvArgs* iv, uint32_t tiles, cudaStream_t st) {
    constexpr int T = 256;
    const size_t sm = ((size_t)fft_cols(L2) << L2) * sizeof(double2);
    if (f) {
        auto k = k_fft_fwd_cols<L2, T>;
        allow_smem(k, sm);
        return launch_k(k, dim3(tiles), dim3(T), sm, st, *f);
    }
    auto k = k_fft_inv_cols<L2, T>;
    allow_smem(k, sm);
    return launch_k(k, dim3(tiles), dim3(T), sm, st, *iv);
}

static cudaError_t fft_dispatch_outer(int l2, const FftFwdArgs* f, const FftInvArgs* iv,
                                      uint32_t tiles, cudaStream_t st) {
    switch (l2) {
        case 2: return fft_outer<2>(f, iv, tiles, st);
        case 3: return fft_outer<3>(f, iv, tiles, st);
        case 4: return fft_outer<4>(f, iv, tiles, st);
        case 5: return fft_outer<5>(f, iv, tiles, st);
        case 6: return fft_outer<6>(f, iv, tiles, st);
        case 7: return fft_outer<7>(f, iv, tiles, st);
        case 8: return fft_outer<8>(f, iv, tiles, st);
        case 9: return fft_outer<9>(f, iv, tiles, st);
        case 10: return fft_outer<10>(f, iv, tiles, st);
        case 11: return fft_outer<11>(f, iv, tiles, st);
        case 12: return fft_outer<12>(f, iv, tiles, st);
        case 13: return fft_outer<13>(f, iv, tiles, st);
        default: return cudaErrorInvalidValue;
    }
}

template <int L1>
static cudaError_t fft_mid(const FftMidArgs& m, uint32_t rows, cudaStream_t st) {
    constexpr int T = fft_row_threads(L1);
    const size_t sm = ((size_t)1 << L1) * sizeof(double2);
    auto k = k_fft_mid_rows<L1, T>;
    allow_smem(k, sm);
    return launch_k(k, dim3(rows), dim3(T), sm, st, m);
}

static cudaError_t fft_dispatch_mid(int l1, const FftMidArgs& m, uint32_t rows, cudaStream_t st) {
    switch (l1) {
        case 3: return fft_mid<3>(m, rows, st);
        case 4: return fft_mid<4>(m, rows, st);
        case 5: return fft_mid<5>(m, rows, st);
        case 6: return fft_mid<6>(m, rows, st);
        case 7: return fft_mid<7>(m, rows, st);
        case 8: return fft_mid<8>(m, rows, st);
        case 9: return fft_mid<9>(m, rows, st);
        case 10: return fft_mid<10>(m, rows, st);
        case 11: return fft_mid<11>(m, rows, st);
        case 12: return fft_mid<12>(m, rows, st);
        case 13: return fft_mid<13>(m, rows, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_fft_product(const uint64_t* a, uint32_t na, const uint64_t* b, uint32_t nb,
                               int bits, int log_n, const FftScratch& s, cudaStream_t st) {
    if (!fft_shape_supported(log_n)) return cudaErrorInvalidValue;
    const FftShape sh = fft_choose_shape(log_n);
    const uint32_t tiles = (1u << sh.log_n1) / fft_cols(sh.log_n2);
    FftFwdArgs f{a, b, na, nb, bits, s.y, log_n, sh.log_n1};
    cudaError_t e = fft_dispatch_outer(sh.log_n2, &f, nullptr, tiles, st);
    if (e != cudaSuccess) return e;
    FftMidArgs m{s.y, log_n, sh.log_n2};
    e = fft_dispatch_mid(sh.log_n1, m, 1u << sh.log_n2, st);
    if (e != cudaSuccess) return e;
    FftInvArgs iv{s.y, s.coef, s.maxerr, log_n, sh.log_n1};
    e = fft_dispatch_outer(sh.log_n2, nullptr, &iv, tiles, st);
    if (e != cudaSuccess) return e;
    FftChunkArgs ck{s.coef, 1u << log_n, bits, s.nchunks, s.chunks, s.spill};
    return launch_k(k_fft_chunks, dim3((s.nchunks + 255) / 256), dim3(256), 0, st, ck);
}

}  // namespace bgpu
