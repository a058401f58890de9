// Three-prime NTT product pipeline for sm_100a.
//
// A product of N = N1 * N2 points (point n = n1 + N1*n2, 32-bit digits) is
// four kernel launches:
//   1. k_fwd_cols   per (8-column tile, prime, operand): load digits straight
//                   from the caller's limbs/Digits, reduce mod p, length-N2
//                   DIF over n2 (natural -> bit-reversed k2), multiply by
//                   omega_N^(n1*k2), store Y[slot][n1].
//   2. k_mid_rows   per (row slot, prime): length-N1 DIF of A's and B's row,
//                   pointwise product (scaled by N^-1), length-N1 DIT back to
//                   natural n1, multiply by omega_N^-(n1*k2), store in place.
//   3. k_inv_cols   per 8-column tile: for each prime, length-N2 DIT over the
//                   bit-reversed slots -> natural n2; then Garner CRT per point
//                   and the sum of each chunk of 8 consecutive coefficients
//                   (an exact 256-bit chunk value plus a < 2^58 spill).
//   4. k_carry      one chunk per thread: chunk + previous spill, carries
//                   resolved by a decoupled look-back scan over blocks, final
//                   limbs or 28-bit digits written in natural order.
// The reference runs the same transform as log2 N barrier-separated radix-2
// sweeps plus a serial carry (src/mul/ntt_multithread.cpp:333-379, 418-442);
// here every pass keeps a whole row or column tile in shared memory and runs
// radix-8/16 rounds in registers, so each product makes three sweeps over the
// residues in global memory.  Template parameter PS selects the prime set
// (arith.cuh): set 0 uses lazy butterflies, set 1 strict ones.
#include <cuda/atomic>

#include <algorithm>

#include "engine.h"
#include "pass_common.cuh"
#include "small_bodies.cuh"

namespace bgpu {

// Row-pass CTAs are held to a register budget below what the compiler takes
// on its own, so that more of them share an SM: rows of 2^10 to 2^12 points at
// 1024 threads' worth per SM (64 registers a thread: sixteen, eight or four
// CTAs), rows of 2^13 points at three 256-thread CTAs (80 registers; their two
// shared row buffers leave room for no more).  Measured per product back to
// back, each against the compiler's own choice or the earlier cap:
//   2^20 points (2^24 x 2^24 bits, rows of 2^11): 61.98 us against 62.16 at
//     1152 threads' worth (56 registers), 63.42 at 1280 (48), 62.87 at 896;
//   2^19 points (rows of 2^10): 38.97 against 39.6 at 1280;
//   2^21 points (rows of 2^12): 119.2 against 126.4 (95 registers, two CTAs),
//     122.3 at three CTAs, 121.4 at five;
//   2^22 points (rows of 2^13): 239.7 against 254.8 (88 registers, two CTAs).
// Longer rows keep the compiler's choice.
#ifndef BGPU_MID_THREADS_PER_SM
#define BGPU_MID_THREADS_PER_SM 1024
#endif
__host__ __device__ constexpr int mid_min_blocks(int l1, int threads) {
    return threads < 64 ? 1 : (l1 <= 12 ? BGPU_MID_THREADS_PER_SM / threads : (l1 == 13 ? 768 / threads : 1));
}

constexpr int kCols = 8;  // columns per outer tile == 32-bit digits per carry chunk
// The forward pass's tiles and threads (measured against 4-column tiles of
// 128 or 64 threads and 8-column tiles of 128 threads: all slower).
constexpr int kFwdCols = 8;
constexpr int kFwdThreads = 256;

__constant__ NttConsts c_consts[kConstSlots];

cudaError_t upload_consts(int slot, const NttConsts& c) {
    return cudaMemcpyToSymbol(c_consts, &c, sizeof(NttConsts), slot * sizeof(NttConsts));
}

// ---- register-resident butterflies ------------------------------------------

// DIF stages for pair bits HI..LO on the 2^R elements base + (j << LO),
// starting at stage T0 (the stages before it already done by the caller).
// Element pair (i, i+h): (a, b) -> (a+b, (a-b) * omega_{2h}^(i mod h)).
template <bool LAZY, int R, int HI, int LO, int T0 = 0>
__device__ __forceinline__ void dif_regs(uint32_t (&x)[1 << R], uint32_t base_low,
                                         const uint2* __restrict__ tw, uint32_t p) {
    const uint2* twb = tw + base_low;  // every twiddle below is twb[compile-time offset]
#pragma unroll
    for (int t = T0; t < R; ++t) {
        const uint32_t h = 1u << (HI - t);
        const int dist = 1 << (R - 1 - t);
#pragma unroll
        for (int j = 0; j < (1 << R); ++j) {
            if (j & dist) continue;
            if (LO == 0 && (j & (dist - 1)) == 0) {
                Bfly<LAZY>::dif1(x[j], x[j + dist], p);  // omega^0 (base_low is 0 when LO == 0)
            } else {
                const uint2 w = __ldg(twb + h + ((uint32_t)(j & (dist - 1)) << LO));
                Bfly<LAZY>::dif(x[j], x[j + dist], w.x, w.y, p);
            }
        }
    }
}

// DIT stages for pair bits LO..HI (inverse table):
// (a, b) -> (a + b*w, a - b*w), w = omega_{2h}^-(i mod h).
template <bool LAZY, int R, int HI, int LO>
__device__ __forceinline__ void dit_regs(uint32_t (&x)[1 << R], uint32_t base_low,
                                         const uint2* __restrict__ tw, uint32_t p) {
    const uint2* twb = tw + base_low;
#pragma unroll
    for (int t = R - 1; t >= 0; --t) {
        const uint32_t h = 1u << (HI - t);
        const int dist = 1 << (R - 1 - t);
#pragma unroll
        for (int j = 0; j < (1 << R); ++j) {
            if (j & dist) continue;
            if (LO == 0 && (j & (dist - 1)) == 0) {
                Bfly<LAZY>::dit1(x[j], x[j + dist], p);
            } else {
                const uint2 w = __ldg(twb + h + ((uint32_t)(j & (dist - 1)) << LO));
                Bfly<LAZY>::dit(x[j], x[j + dist], w.x, w.y, p);
            }
        }
    }
}

// One smem round (load -> butterflies -> store back); no sync inside.
template <bool LAZY, int L, int C, int T, int K, bool INV>
__device__ __forceinline__ void smem_round(uint32_t* sm, const uint2* __restrict__ tw, uint32_t p,
                                           int tid) {
    using Gr = Group<L, C, K>;
    constexpr int R = Gr::R;
#pragma unroll 2
    for (int g = tid; g < Gr::G; g += T) {
        const Gr gr(g);
        uint32_t x[1 << R];
#pragma unroll
        for (int j = 0; j < (1 << R); ++j) x[j] = sm[gr.at(j)];
        if constexpr (INV)
            dit_regs<LAZY, R, Gr::HI, Gr::LO>(x, gr.base_low, tw, p);
        else
            dif_regs<LAZY, R, Gr::HI, Gr::LO>(x, gr.base_low, tw, p);
#pragma unroll
        for (int j = 0; j < (1 << R); ++j) sm[gr.at(j)] = x[j];
    }
}

// DIF rounds K..KEND in smem, each followed by a block barrier.
template <bool LAZY, int L, int C, int T, int K, int KEND>
__device__ __forceinline__ void dif_rounds(uint32_t* sm, const uint2* tw, uint32_t p, int tid) {
    if constexpr (K <= KEND) {
        smem_round<LAZY, L, C, T, K, false>(sm, tw, p, tid);
        __syncthreads();
        dif_rounds<LAZY, L, C, T, K + 1, KEND>(sm, tw, p, tid);
    }
}

// DIT rounds K down to KEND in smem, each followed by a barrier.
template <bool LAZY, int L, int C, int T, int K, int KEND>
__device__ __forceinline__ void dit_rounds(uint32_t* sm, const uint2* tw, uint32_t p, int tid) {
    if constexpr (K >= KEND) {
        smem_round<LAZY, L, C, T, K, true>(sm, tw, p, tid);
        __syncthreads();
        dit_rounds<LAZY, L, C, T, K - 1, KEND>(sm, tw, p, tid);
    }
}

// omega_N^(+-e) as a fully reduced Montgomery form from the two split tables.
__device__ __forceinline__ uint32_t inter_twiddle(const NttConsts& c, int q, int dir, uint32_t e,
                                                  int log_n, uint32_t p) {
    const uint32_t em = e << (c.log_max - log_n);
    const uint32_t hi = __ldg(&c.th[q][dir][em >> c.split].x);
    const uint2 lo = __ldg(&c.tl[q][dir][em & ((1u << c.split) - 1u)]);
    return mont_mul_pre(hi, lo.x, lo.y, p);
}

// x * omega (omega from inter_twiddle), lazily (0, 2p) or strictly [0, p).
template <bool LAZY>
__device__ __forceinline__ uint32_t twiddle_mul(uint32_t x, uint32_t w, uint32_t p, uint32_t pinv) {
    const uint32_t r = mont_lazy(x, w, w * pinv, p);
    return LAZY ? r : csub(r, p);
}

// x * S * B for Montgomery pairs S = (w, w') and B = (bw, bw'): the
// inter-pass twiddle split as a per-CTA power table entry times a per-group
// factor, lazily (0, 2p) or strictly [0, p).
template <bool LAZY>
__device__ __forceinline__ uint32_t mul2(uint32_t x, uint2 sp, uint32_t bw, uint32_t bwp,
                                         uint32_t p) {
    const uint32_t y = mont_lazy(mont_lazy(x, sp.x, sp.y, p), bw, bwp, p);
    return LAZY ? y : csub(y, p);
}

__host__ __device__ constexpr uint32_t brev_c(uint32_t v, int bits) {
    uint32_t r = 0;
    for (int i = 0; i < bits; ++i) r |= ((v >> i) & 1u) << (bits - 1 - i);
    return r;
}

__device__ __forceinline__ uint32_t bitrev(uint32_t v, int bits) {
    return bits == 0 ? 0u : (__brev(v) >> (32 - bits));
}


// ---- kernel 1: forward column pass ------------------------------------------


// Returned by value: binding a reference to the kernel parameter would force
// a copy of it into local memory.
__device__ __forceinline__ ProductDesc product(const ProductDesc* descs, const ProductDesc& one,
                                              uint32_t p) {
    return descs ? descs[p] : one;
}

// 32-bit digit n of an operand in a format known at compile time (0 beyond
// its length).
template <bool LIMB>
__device__ __forceinline__ uint32_t load_digit32_fmt(const OperandDesc& in, uint32_t n) {
    if (n >= in.nd32) return 0u;
    if constexpr (LIMB) {
        return __ldg(static_cast<const uint32_t*>(in.ptr) + n);
    } else {
        const uint32_t* d = static_cast<const uint32_t*>(in.ptr);
        const uint32_t bit = n * 32u;
        const uint32_t i0 = bit / 28u, sh = bit - i0 * 28u;  // sh in {0,4,...,24}
        uint32_t v = __ldg(d + i0) >> sh;
        if (i0 + 1 < in.nsrc) v |= __ldg(d + i0 + 1) << (28u - sh);
        return v;
    }
}

// Round 0 of the forward column pass: rows n2 = base + (j << LO) read from
// the caller's digits (u64 limbs when LIMB, else 28-bit Digits), reduced into
// [0, 2p) ([0, p) for the strict set) and transformed.  HALF: the operand
// fills at most the lower half of the transform, so the elements of the upper
// half (j >= 2^(R-1), rows n2 >= N2/2) are zero: they are not loaded, and the
// first stage (a, 0) -> (a, a w) is one multiply per pair.  With a single
// round the inter-pass twiddle and the global store follow; otherwise the
// elements go to the shared tile.
template <int PS, int L2, int T, int FC, bool LIMB, bool HALF>
__device__ __forceinline__ void fwd_round0(const FwdColsArgs& a, const OperandDesc& in, const NttConsts& c,
                                           int q, uint32_t c0, uint32_t* y, const uint2* sS, uint32_t* sm) {
    constexpr bool LAZY = PS == 0;
    using P2 = Plan<L2>;
    constexpr int NR = P2::nr;
    constexpr int RL = P2::r(NR - 1);
    constexpr int SROW = (1 << RL) + 1;
    using Gr = Group<L2, FC, 0>;
    constexpr int R = Gr::R;
    constexpr int D = 1 << (R - 1);
    constexpr int NL = HALF ? D : (1 << R);  // elements read from the operand
    const uint32_t p = c.pr[q].p, pinv = c.pr[q].pinv, red = c.red[q];
    const uint2* tw = c.stage[q][0];
    const uint32_t stride = 1u << (Gr::LO + a.log_n1);  // digit step between a group's rows
#pragma unroll 2
    for (int g = threadIdx.x; g < Gr::G; g += T) {
        const Gr gr(g);
        uint32_t x[1 << R];
        uint32_t any = 0;
        uint32_t n = c0 + gr.col + (gr.base << a.log_n1);
#pragma unroll
        for (int j = 0; j < NL; ++j, n += stride) {
            const uint32_t v = load_digit32_fmt<LIMB>(in, n);
            any |= v;
            // v - floor(v * red / 2^32) * p lies in [0, 2p) for any 32-bit v
            const uint32_t r = v - __umulhi(v, red) * p;
            x[j] = LAZY ? r : csub(r, p);
        }
        if (any) {
            if constexpr (HALF) {
                const uint2* twb = tw + gr.base_low;
#pragma unroll
                for (int j = 0; j < D; ++j) {
                    if (Gr::LO == 0 && j == 0) {
                        x[j + D] = x[j];  // omega^0 (base_low is 0 when LO == 0)
                    } else {
                        const uint2 w = __ldg(twb + (1u << Gr::HI) + ((uint32_t)j << Gr::LO));
                        const uint32_t t = shoup_lazy(x[j], w.x, w.y, p);
                        x[j + D] = LAZY ? t : csub(t, p);
                    }
                }
                dif_regs<LAZY, R, Gr::HI, Gr::LO, 1>(x, gr.base_low, tw, p);
            } else {
                dif_regs<LAZY, R, Gr::HI, Gr::LO>(x, gr.base_low, tw, p);
            }
        } else {
#pragma unroll
            for (int j = 0; j < (1 << R); ++j) x[j] = 0;
        }
        if constexpr (NR == 1) {
            const uint32_t n1 = c0 + gr.col;
            const uint32_t bw = inter_twiddle(c, q, 0, (n1 * bitrev(gr.base, L2)) & ((1u << a.log_n) - 1u),
                                              a.log_n, p);
            const uint32_t bwp = bw * pinv;
            const uint2* srow = sS + gr.col * SROW;
#pragma unroll
            for (int j = 0; j < (1 << R); ++j)
                y[(gr.idx(j) << a.log_n1) + n1] = mul2<LAZY>(x[j], srow[brev_c(j, R)], bw, bwp, p);
        } else {
#pragma unroll
            for (int j = 0; j < (1 << R); ++j) sm[gr.at(j)] = x[j];
        }
    }
}

// Column tiles of 2^9 rows run 8 CTAs of 256 threads per SM (32 registers a
// thread, a few bytes spilled): measured at 2^20 points, the product is
// 0.4 us shorter than with the 40 registers the compiler picks on its own
// (6 CTAs per SM).  Tiles of 2^10 rows run 4 CTAs (64 registers, no spills)
// where the compiler took 124 registers for 2: at 2^23 points (2^27 x 2^27
// bits) 502.8 -> 476.0 us per product (3 CTAs at 80 registers: 486.4).
// Tiles of 2^11 rows keep the compiler's choice (3 CTAs at 80 registers,
// all their shared memory allows, measured no faster: 1126.3 against
// 1125.6 us at 2^24 points); so do the shorter ones.
__host__ __device__ constexpr int fwd_min_blocks(int l2, int threads) {
    return l2 == 9 ? 2048 / threads : (l2 == 10 ? 1024 / threads : 1);
}

// The forward column pass of one CTA: tile bx, prime by, operand and product
// bz (block coordinates passed in, so a mixed-length launch can run it too).
template <int PS, int L2, int T, int FC = kCols>
__device__ __forceinline__ void fwd_cols_body(const FwdColsArgs& a, uint32_t bx, uint32_t by, uint32_t bz,
                                              uint32_t* sm) {  // sm: [2^L2][FC] + column powers
    constexpr bool LAZY = PS == 0;
    using P2 = Plan<L2>;
    constexpr int NR = P2::nr;
    const NttConsts& c = c_consts[a.slot];
    const int q = (int)by, opi = (int)(bz % (uint32_t)a.nops);
    const ProductDesc pd = product(a.descs, a.one, bz / (uint32_t)a.nops);
    const uint32_t p = c.pr[q].p, pinv = c.pr[q].pinv;
    const uint2* tw = c.stage[q][0];
    const OperandDesc in = opi == 0 ? pd.op[0] : pd.op[1];
    const uint32_t c0 = bx * FC;
    const size_t nn = (size_t)1 << a.log_n;
    uint32_t* y = pd.y + ((size_t)opi * kNumPrimes + q) * nn;

    // The last round's groups hold slots base + j (LO = 0) of one column n1;
    // k2 = bitrev(base) + bitrev_RL(j) << (L2-RL), so the inter-pass twiddle
    // omega_N^(n1*k2) = B(group) * S_col^bitrev_RL(j).  sS[col][m] holds the
    // column powers S_col^m = omega_N^(n1 * m << (L2-RL)).  Rows are padded to
    // 2^RL + 1 entries so the 8 columns a warp reads at one m sit in distinct
    // banks (an unpadded 2^RL-entry row puts all of them in one bank).
    constexpr int RL = P2::r(NR - 1);
    constexpr int SROW = (1 << RL) + 1;
    uint2* sS = reinterpret_cast<uint2*>(sm + (FC << L2));
    for (int t = threadIdx.x; t < (FC << RL); t += T) {
        const uint32_t col = (uint32_t)t >> RL, m = (uint32_t)t & ((1u << RL) - 1u);
        const uint32_t e = (((c0 + col) * m) << (L2 - RL)) & (uint32_t)(nn - 1);
        const uint32_t w = inter_twiddle(c, q, 0, e, a.log_n, p);
        sS[col * SROW + m] = make_uint2(w, w * pinv);
    }
    if constexpr (NR == 1) __syncthreads();
    if (!a.overlap) pdl_wait();

    // Round 0: rows n2 = base + (j << LO) read from the caller's digits.
    // The digit format and whether the operand fills at most the lower half
    // of the transform (then every row n2 >= N2/2 is zero) are uniform over
    // the launch, so each combination is its own copy of the round.
    if (in.fmt == kFmtLimb64) {
        if (2 * (size_t)in.nd32 <= nn)
            fwd_round0<PS, L2, T, FC, true, true>(a, in, c, q, c0, y, sS, sm);
        else
            fwd_round0<PS, L2, T, FC, true, false>(a, in, c, q, c0, y, sS, sm);
    } else {
        if (2 * (size_t)in.nd32 <= nn)
            fwd_round0<PS, L2, T, FC, false, true>(a, in, c, q, c0, y, sS, sm);
        else
            fwd_round0<PS, L2, T, FC, false, false>(a, in, c, q, c0, y, sS, sm);
    }
    if constexpr (NR > 1) {
        __syncthreads();
        dif_rounds<LAZY, L2, FC, T, 1, NR - 2>(sm, tw, p, threadIdx.x);
        // Last round: butterflies, inter-pass twiddle, store to global.
        using Gr = Group<L2, FC, NR - 1>;
        constexpr int R = Gr::R;
#pragma unroll 2
        for (int g = threadIdx.x; g < Gr::G; g += T) {
            const Gr gr(g);
            uint32_t x[1 << R];
#pragma unroll
            for (int j = 0; j < (1 << R); ++j) x[j] = sm[gr.at(j)];
            dif_regs<LAZY, R, Gr::HI, Gr::LO>(x, gr.base_low, tw, p);
            const uint32_t n1 = c0 + gr.col;
            const uint32_t bw = inter_twiddle(c, q, 0, (n1 * bitrev(gr.base, L2)) & (uint32_t)(nn - 1),
                                              a.log_n, p);
            const uint32_t bwp = bw * pinv;
            const uint2* srow = sS + gr.col * SROW;
#pragma unroll
            for (int j = 0; j < (1 << R); ++j)
                y[(gr.idx(j) << a.log_n1) + n1] = mul2<LAZY>(x[j], srow[brev_c(j, R)], bw, bwp, p);
        }
    }
    // Let the row pass launch only once this CTA's work is done: an early
    // trigger parks row-pass CTAs on SMs the column pass still fills.
    pdl_trigger();
    if (a.overlap) pdl_wait();
}

template <int PS, int L2, int T>
__global__ void __launch_bounds__(T, fwd_min_blocks(L2, T)) k_fwd_cols(const FwdColsArgs a) {
    extern __shared__ __align__(16) uint32_t sm[];
    fwd_cols_body<PS, L2, T, kFwdCols>(a, blockIdx.x, blockIdx.y, blockIdx.z, sm);
}

// ---- kernel 2: middle row pass ----------------------------------------------


// a*b*2^-32 mod p in [0, p); the 2^-32 and the inverse transform's N^-1 are
// both cancelled by the scale N^-1 * 2^32 folded into the row's inverse
// inter-pass twiddle (one multiply per group instead of one per point).
template <bool LAZY>
__device__ __forceinline__ uint32_t pointwise(uint32_t a, uint32_t b, uint32_t p, uint32_t pinv) {
    if constexpr (LAZY)
        return csub(mont_lazy(a, b, b * pinv, p), p);  // a, b < 2p, 4p < 2^32: product term < p
    else
        return mont_mul(a, b, p, pinv);
}

// Rows too long for two row buffers in shared memory (2^15 points of a
// non-square product): A's transformed row is parked in its own global plane
// and read back there by the pointwise product, while B's row uses the one
// shared buffer.
template <int L1, bool SQR>
constexpr bool kOneRowBuffer = !SQR && L1 >= 15;

// Thread number within a row's group of T threads: the CTA's own thread
// number when the CTA is one group (MULTI false: the compiler re-reads it
// instead of holding a computed copy in a register), else the position in
// its group (a CTA holding several rows of a mixed-length launch).
template <int T, bool MULTI>
__device__ __forceinline__ int sub_tid() {
    return MULTI ? (int)(threadIdx.x & (T - 1)) : (int)threadIdx.x;
}

// Last DIF round of B (or A when squaring) fused with the pointwise product
// and the first DIT round; with a single round also the inverse twiddle.
template <bool LAZY, int L1, int T, bool SQR, bool SINGLE, bool MULTI>
__device__ __forceinline__ void mid_turn(const MidRowsArgs& a, const NttConsts& c, uint32_t* sa,
                                         uint32_t* sb, const uint32_t* row_a, const uint32_t* row_b,
                                         uint32_t* row_out, int q, uint32_t k2, const uint2* sT) {
    const int tid = sub_tid<T, MULTI>();
    constexpr bool ONE = kOneRowBuffer<L1, SQR>;
    using P1 = Plan<L1>;
    constexpr int K = P1::nr - 1;
    using Gr = Group<L1, 1, K>;
    constexpr int R = Gr::R;
    const uint32_t p = c.pr[q].p, pinv = c.pr[q].pinv;
    const uint2* twf = c.stage[q][0];
    const uint2* twi = c.stage[q][1];
    const uint32_t sw = q == 0 ? a.scale_w[0] : (q == 1 ? a.scale_w[1] : a.scale_w[2]);
    const uint32_t swp = q == 0 ? a.scale_wp[0] : (q == 1 ? a.scale_wp[1] : a.scale_wp[2]);
    const uint32_t* src = (SQR || ONE) ? sa : sb;
#pragma unroll 1
    for (int g = tid; g < Gr::G; g += T) {
        const Gr gr(g);
        uint32_t x[1 << R];
#pragma unroll
        for (int j = 0; j < (1 << R); ++j) {
            if constexpr (SINGLE)
                x[j] = (SQR ? row_a : row_b)[gr.idx(j)];
            else
                x[j] = src[gr.at(j)];
        }
        dif_regs<LAZY, R, Gr::HI, Gr::LO>(x, gr.base_low, twf, p);
#pragma unroll
        for (int j = 0; j < (1 << R); ++j) {
            const uint32_t other = SQR ? x[j] : (ONE ? row_a[gr.idx(j)] : sa[gr.at(j)]);
            x[j] = pointwise<LAZY>(x[j], other, p, pinv);
        }
        dit_regs<LAZY, R, Gr::HI, Gr::LO>(x, gr.base_low, twi, p);
        if constexpr (SINGLE) {
            // one round covers the row: n1 = j, twiddle omega^-(k2 j) = sT[j]
            const uint32_t bw = sw, bwp = swp;  // the scale N^-1 * 2^32 (no inter-pass twiddle part)
#pragma unroll
            for (int j = 0; j < (1 << R); ++j) row_out[gr.idx(j)] = mul2<LAZY>(x[j], sT[j], bw, bwp, p);
        } else {
#pragma unroll
            for (int j = 0; j < (1 << R); ++j) sa[gr.at(j)] = x[j];
        }
    }
}

// DIF of one row: round 0 from global into smem, then rounds 1..nr-2 (the
// last round is done by mid_turn).
template <bool LAZY, int L1, int T, bool MULTI>
__device__ __forceinline__ void mid_dif_row(const uint32_t* row, uint32_t* s, const uint2* twf,
                                            uint32_t p) {
    const int tid = sub_tid<T, MULTI>();
    using P1 = Plan<L1>;
    using Gr = Group<L1, 1, 0>;
    constexpr int R = Gr::R;
#pragma unroll 2
    for (int g = tid; g < Gr::G; g += T) {
        const Gr gr(g);
        uint32_t x[1 << R];
#pragma unroll
        for (int j = 0; j < (1 << R); ++j) x[j] = row[gr.idx(j)];
        dif_regs<LAZY, R, Gr::HI, Gr::LO>(x, gr.base_low, twf, p);
#pragma unroll
        for (int j = 0; j < (1 << R); ++j) s[gr.at(j)] = x[j];
    }
    __syncthreads();
    dif_rounds<LAZY, L1, 1, T, 1, P1::nr - 2>(s, twf, p, tid);
}

// The last DIT round's groups hold n1 = q + (j << LO0); the inverse
// inter-pass twiddle omega_N^-(k2 n1) = B(q) * T^j with the row-constant
// powers sT[j] = omega_N^-(k2 j << LO0), written here for one row.
template <int L1, int T>
__device__ __forceinline__ void row_inv_powers(const NttConsts& c, int q, uint32_t k2, int log_n, size_t nn,
                                               uint32_t p, uint32_t pinv, uint2* sT, int tid) {
    using P1 = Plan<L1>;
    constexpr int R0 = P1::r(0), LO0 = P1::lo(0);
    for (int t = tid; t < (1 << R0); t += T) {
        const uint32_t w = inter_twiddle(c, q, 1, ((k2 * (uint32_t)t) << LO0) & (uint32_t)(nn - 1), log_n, p);
        sT[t] = make_uint2(w, w * pinv);
    }
}

// Round 0 of a row's DIT (its top bits) from shared memory `s`; each group
// times its inverse inter-pass twiddle and the scale N^-1 * 2^32 (sw, swp),
// stored to the row in global memory.
template <bool LAZY, int L1, int T>
__device__ __forceinline__ void row_dit_store(const NttConsts& c, int q, uint32_t k2, int log_n, size_t nn,
                                              uint32_t sw, uint32_t swp, const uint32_t* s, const uint2* sT,
                                              const uint2* twi, uint32_t p, uint32_t pinv, uint32_t* row,
                                              int tid) {
    using Gr = Group<L1, 1, 0>;
    constexpr int R = Gr::R;
#pragma unroll 2
    for (int g = tid; g < Gr::G; g += T) {
        const Gr gr(g);
        uint32_t x[1 << R];
#pragma unroll
        for (int j = 0; j < (1 << R); ++j) x[j] = s[gr.at(j)];
        dit_regs<LAZY, R, Gr::HI, Gr::LO>(x, gr.base_low, twi, p);
        const uint32_t bw =
            mont_mul_pre(inter_twiddle(c, q, 1, (k2 * gr.base) & (uint32_t)(nn - 1), log_n, p), sw, swp, p);
        const uint32_t bwp = bw * pinv;
#pragma unroll
        for (int j = 0; j < (1 << R); ++j) row[gr.idx(j)] = mul2<LAZY>(x[j], sT[j], bw, bwp, p);
    }
}

// The row pass of one row: row slot `slot`, prime and product from `by`
// (prime + 3 * product), run by T threads on the shared slice `sm`; every
// thread of the CTA takes the same barriers, so a CTA may hold several rows
// of the same length side by side (MULTI).
template <int PS, int L1, int T, bool SQR, bool MULTI = false>
__device__ __forceinline__ void mid_rows_body(const MidRowsArgs& a, uint32_t slot, uint32_t by,
                                              uint32_t* sm) {  // sm: sa[2^L1] (+ sb[2^L1]) + powers
    constexpr bool LAZY = PS == 0;
    constexpr bool ONE = kOneRowBuffer<L1, SQR>;
    const int tid = sub_tid<T, MULTI>();
    using P1 = Plan<L1>;
    constexpr int NR = P1::nr;
    static_assert(!ONE || NR > 1, "the one-buffer row pass needs several rounds");
    const NttConsts& c = c_consts[a.slot];
    uint32_t* sa = sm;
    uint32_t* sb = sm + (1u << L1);
    const int q = (int)(by % kNumPrimes);
    const ProductDesc pd = product(a.descs, a.one, by / kNumPrimes);
    const uint32_t p = c.pr[q].p, pinv = c.pr[q].pinv;
    const uint2* twf = c.stage[q][0];
    const uint2* twi = c.stage[q][1];
    const size_t nn = (size_t)1 << a.log_n;
    uint32_t* row_a = pd.y + q * nn + (size_t)slot * (1u << L1);
    const uint32_t* row_b = SQR ? nullptr : pd.y + (kNumPrimes + q) * nn + (size_t)slot * (1u << L1);
    const uint32_t k2 = bitrev(slot, a.log_n2);
    const uint32_t sw = q == 0 ? a.scale_w[0] : (q == 1 ? a.scale_w[1] : a.scale_w[2]);
    const uint32_t swp = q == 0 ? a.scale_wp[0] : (q == 1 ? a.scale_wp[1] : a.scale_wp[2]);

    // The last DIT round's groups hold n1 = q + (j << LO0); the inverse
    // inter-pass twiddle omega_N^-(k2 n1) = B(q) * T^j with the row-constant
    // powers sT[j] = omega_N^-(k2 j << LO0).  (row_inv_powers and
    // row_dit_store do the same steps for the spectral row passes; they are
    // written out here because routing this body through them changed the
    // register allocation, and the spills, of the mixed-length row launch
    // that inlines it.)
    constexpr int R0 = P1::r(0), LO0 = P1::lo(0);
    uint2* sT = reinterpret_cast<uint2*>(sm + ((SQR || ONE ? 1u : 2u) << L1));
    for (int t = tid; t < (1 << R0); t += T) {
        const uint32_t w = inter_twiddle(c, q, 1, ((k2 * (uint32_t)t) << LO0) & (uint32_t)(nn - 1),
                                         a.log_n, p);
        sT[t] = make_uint2(w, w * pinv);
    }
    __syncthreads();
    pdl_wait();

    if constexpr (NR == 1) {
        if constexpr (!SQR) {
            using Gr = Group<L1, 1, 0>;
            constexpr int R = Gr::R;
#pragma unroll 1
            for (int g = tid; g < Gr::G; g += T) {
                const Gr gr(g);
                uint32_t x[1 << R];
#pragma unroll
                for (int j = 0; j < (1 << R); ++j) x[j] = row_a[gr.idx(j)];
                dif_regs<LAZY, R, Gr::HI, Gr::LO>(x, gr.base_low, twf, p);
#pragma unroll
                for (int j = 0; j < (1 << R); ++j) sa[gr.at(j)] = x[j];
            }
            __syncthreads();
        }
        mid_turn<LAZY, L1, T, SQR, true, MULTI>(a, c, sa, sb, row_a, row_b, row_a, q, k2, sT);
    } else {
        mid_dif_row<LAZY, L1, T, MULTI>(row_a, sa, twf, p);
        if constexpr (ONE) {
            smem_round<LAZY, L1, 1, T, NR - 1, false>(sa, twf, p, tid);  // A's last DIF round
            __syncthreads();
            // park A's transform in its plane (element i at row_a[i]) ...
            for (uint32_t i = tid; i < (1u << L1); i += T) row_a[i] = sa[sidx<1>(i, 0)];
            __syncthreads();
            // ... and transform B in the same buffer
            mid_dif_row<LAZY, L1, T, MULTI>(row_b, sa, twf, p);
        } else if constexpr (!SQR) {
            smem_round<LAZY, L1, 1, T, NR - 1, false>(sa, twf, p, tid);  // A's last DIF round
            mid_dif_row<LAZY, L1, T, MULTI>(row_b, sb, twf, p);
        }
        mid_turn<LAZY, L1, T, SQR, false, MULTI>(a, c, sa, sb, row_a, row_b, row_a, q, k2, sT);
        __syncthreads();
        dit_rounds<LAZY, L1, 1, T, NR - 2, 1>(sa, twi, p, tid);
        // Round 0 (top bits): DIT, inverse twiddle, store to global.
        using Gr = Group<L1, 1, 0>;
        constexpr int R = Gr::R;
#pragma unroll 2
        for (int g = tid; g < Gr::G; g += T) {
            const Gr gr(g);
            uint32_t x[1 << R];
#pragma unroll
            for (int j = 0; j < (1 << R); ++j) x[j] = sa[gr.at(j)];
            dit_regs<LAZY, R, Gr::HI, Gr::LO>(x, gr.base_low, twi, p);
            // inverse inter-pass twiddle of the group times the scale N^-1 * 2^32
            const uint32_t bw = mont_mul_pre(
                inter_twiddle(c, q, 1, (k2 * gr.base) & (uint32_t)(nn - 1), a.log_n, p), sw, swp, p);
            const uint32_t bwp = bw * pinv;
#pragma unroll
            for (int j = 0; j < (1 << R); ++j) row_a[gr.idx(j)] = mul2<LAZY>(x[j], sT[j], bw, bwp, p);
        }
    }
    pdl_trigger();  // late, as in the column pass
}

template <int PS, int L1, int T, bool SQR>
__global__ void __launch_bounds__(T, mid_min_blocks(L1, T)) k_mid_rows(const MidRowsArgs a) {
    extern __shared__ __align__(16) uint32_t sm[];
    mid_rows_body<PS, L1, T, SQR>(a, blockIdx.x, blockIdx.y, sm);
}

// ---- spectral sums: the row pass split at the pointwise product ----------------
//
// k_rows_dif finishes an operand block's forward transform: the row DIF of
// row blockIdx.x, prime blockIdx.y, stored back in place with element i at
// row[i] (the order the one-buffer row pass parks A's transform in).
// k_rows_mac forms, per row, sum_t sa[t] (.) sb[t] over the launch's pairs of
// such spectra (Montgomery products, so the sum carries 2^-32, which the scale
// in the last round cancels) and runs the row DIT with the inverse
// inter-pass twiddle into y, where the inverse column pass reads it.

template <int PS, int L1, int T>
__global__ void __launch_bounds__(T) k_rows_dif(const SpecArgs a) {
    extern __shared__ __align__(16) uint32_t sm[];  // one row
    constexpr bool LAZY = PS == 0;
    constexpr int NR = Plan<L1>::nr;
    static_assert(NR > 1, "the spectral row passes need several rounds");
    const NttConsts& c = c_consts[a.slot];
    const int q = (int)blockIdx.y;
    const uint32_t p = c.pr[q].p;
    const uint2* twf = c.stage[q][0];
    uint32_t* row = a.y + (size_t)q * ((size_t)1 << a.log_n) + ((size_t)blockIdx.x << L1);
    pdl_wait();
    mid_dif_row<LAZY, L1, T, false>(row, sm, twf, p);
    smem_round<LAZY, L1, 1, T, NR - 1, false>(sm, twf, p, threadIdx.x);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < (1u << L1); i += T) row[i] = sm[sidx<1>(i, 0)];
    pdl_trigger();
}

// NT > 0: exactly NT terms, every term's loads of a group issued before its
// products; NT == 0: any count up to kMaxSpecTerms, one term at a time.
template <int PS, int L1, int T, int NT>
__global__ void __launch_bounds__(T) k_rows_mac(const SpecArgs a) {
    extern __shared__ __align__(16) uint32_t sm[];  // one row + the row's inverse powers
    constexpr bool LAZY = PS == 0;
    constexpr int NR = Plan<L1>::nr;
    static_assert(NR > 1, "the spectral row passes need several rounds");
    const NttConsts& c = c_consts[a.slot];
    const int q = (int)blockIdx.y;
    const uint32_t p = c.pr[q].p, pinv = c.pr[q].pinv;
    const uint2* twi = c.stage[q][1];
    const size_t nn = (size_t)1 << a.log_n;
    const size_t off = (size_t)q * nn + ((size_t)blockIdx.x << L1);
    const uint32_t k2 = bitrev(blockIdx.x, a.log_n2);
    const uint32_t sw = q == 0 ? a.scale_w[0] : (q == 1 ? a.scale_w[1] : a.scale_w[2]);
    const uint32_t swp = q == 0 ? a.scale_wp[0] : (q == 1 ? a.scale_wp[1] : a.scale_wp[2]);
    uint2* sT = reinterpret_cast<uint2*>(sm + (1u << L1));
    row_inv_powers<L1, T>(c, q, k2, a.log_n, nn, p, pinv, sT, threadIdx.x);
    __syncthreads();
    pdl_wait();
    {  // the sum of products, then the first DIT round (the last DIF round's groups)
        using Gr = Group<L1, 1, NR - 1>;
        constexpr int R = Gr::R;
#pragma unroll 2
        for (int g = threadIdx.x; g < Gr::G; g += T) {
            const Gr gr(g);
            uint32_t x[1 << R];
            if constexpr (NT > 0) {
                // the last round's groups are 2^R consecutive elements from
                // a multiple of 2^R (its LO is 0): 16-byte loads
                static_assert(Gr::LO == 0 && R >= 2, "vector loads need whole 4-element runs");
                uint32_t va[NT][1 << R], vb[NT][1 << R];
#pragma unroll
                for (int t = 0; t < NT; ++t) {
                    const uint4* pa = reinterpret_cast<const uint4*>(a.sa[t] + off + gr.base);
                    const uint4* pb = reinterpret_cast<const uint4*>(a.sb[t] + off + gr.base);
#pragma unroll
                    for (int v = 0; v < (1 << R) / 4; ++v) {
                        const uint4 wa = pa[v], wb = pb[v];
                        va[t][4 * v] = wa.x, va[t][4 * v + 1] = wa.y, va[t][4 * v + 2] = wa.z, va[t][4 * v + 3] = wa.w;
                        vb[t][4 * v] = wb.x, vb[t][4 * v + 1] = wb.y, vb[t][4 * v + 2] = wb.z, vb[t][4 * v + 3] = wb.w;
                    }
                }
#pragma unroll
                for (int j = 0; j < (1 << R); ++j) {
                    x[j] = pointwise<LAZY>(va[0][j], vb[0][j], p, pinv);
#pragma unroll
                    for (int t = 1; t < NT; ++t) x[j] = mod_add(x[j], pointwise<LAZY>(va[t][j], vb[t][j], p, pinv), p);
                }
            } else {
#pragma unroll
                for (int j = 0; j < (1 << R); ++j) x[j] = 0;
#pragma unroll
                for (int t = 0; t < kMaxSpecTerms; ++t) {  // constant indices into the parameters
                    if (t >= a.nterms) break;
                    const uint32_t* ra = a.sa[t] + off;
                    const uint32_t* rb = a.sb[t] + off;
#pragma unroll
                    for (int j = 0; j < (1 << R); ++j)
                        x[j] = mod_add(x[j], pointwise<LAZY>(ra[gr.idx(j)], rb[gr.idx(j)], p, pinv), p);
                }
            }
            dit_regs<LAZY, R, Gr::HI, Gr::LO>(x, gr.base_low, twi, p);
#pragma unroll
            for (int j = 0; j < (1 << R); ++j) sm[gr.at(j)] = x[j];
        }
    }
    __syncthreads();
    dit_rounds<LAZY, L1, 1, T, NR - 2, 1>(sm, twi, p, threadIdx.x);
    row_dit_store<LAZY, L1, T>(c, q, k2, a.log_n, nn, sw, swp, sm, sT, twi, p, pinv, a.y + off, threadIdx.x);
    pdl_trigger();
}

// ---- kernel 3: inverse column pass + CRT + chunk sums -------------------------


// Garner: residues (r0,r1,r2), each in [0, p_q) -> the coefficient as 96 bits.
__device__ __forceinline__ void crt3(const NttConsts& c, uint32_t r0, uint32_t r1, uint32_t r2,
                                     uint32_t& w0, uint32_t& w1, uint32_t& w2) {
    const uint32_t p1 = c.pr[1].p, p2 = c.pr[2].p, p0 = c.pr[0].p;
    const uint32_t t1 = mont_mul_pre(mod_sub(r1, r0, p1), c.k1, c.k1p, p1);   // (r1-r0)/p0 mod p1
    const uint32_t d2 = mod_sub(r2, r0, p2);
    const uint32_t e2 = mont_mul_pre(t1, c.k2, c.k2p, p2);                    // p0*t1 mod p2
    const uint32_t t2 = mont_mul_pre(mod_sub(d2, e2, p2), c.k3, c.k3p, p2);   // /(p0 p1) mod p2
    // v = r0 + p0*t1 + p0*p1*t2
    const uint64_t a = (uint64_t)p0 * t1 + r0;
    const uint64_t blo = c.m01 * (uint64_t)t2;
    const uint64_t bhi = __umul64hi(c.m01, (uint64_t)t2);
    const uint64_t lo = a + blo;
    const uint64_t hi = bhi + (lo < a ? 1u : 0u);
    w0 = (uint32_t)lo;
    w1 = (uint32_t)(lo >> 32);
    w2 = (uint32_t)hi;
}

#ifndef BGPU_INV_UNROLL
#define BGPU_INV_UNROLL 4
#endif

constexpr int kInvUnroll = BGPU_INV_UNROLL;  // groups of the first (global-memory) round in flight per thread

// The inverse column pass of one CTA: tile bx of product by.  Three thread
// groups of TP threads, one per prime, transform their prime's column tile
// side by side; then all threads do the CRT.
template <int PS, int L2, int TP>
__device__ __forceinline__ void inv_cols_body(const InvColsArgs& a, uint32_t bx, uint32_t by,
                                              uint32_t* sm) {  // sm: 3 x [2^L2][kCols]
    constexpr bool LAZY = PS == 0;
    constexpr int T = kNumPrimes * TP;
    using P2 = Plan<L2>;
    constexpr int NR = P2::nr;
    constexpr int TILE = kCols << L2;
    const NttConsts& c = c_consts[a.slot];
    const uint32_t n1_len = 1u << a.log_n1, c0 = bx * kCols;
    const size_t nn = (size_t)1 << a.log_n;
    const int q = threadIdx.x / TP, tq = threadIdx.x % TP;
    const ProductDesc pd = product(a.descs, a.one, by);
    uint32_t* s = sm + q * TILE;
    const uint32_t p = c.pr[q].p;
    const uint2* twi = c.stage[q][1];
    const uint32_t* z = pd.y + q * nn;
    pdl_wait();
    pdl_trigger();
    // Round NR-1 (lowest bits): load slots from global.
    {
        using Gr = Group<L2, kCols, NR - 1>;
        constexpr int R = Gr::R;
#pragma unroll kInvUnroll
        for (int g = tq; g < Gr::G; g += TP) {
            const Gr gr(g);
            uint32_t x[1 << R];
#pragma unroll
            for (int j = 0; j < (1 << R); ++j)
                x[j] = z[(gr.idx(j) << a.log_n1) + c0 + gr.col];
            dit_regs<LAZY, R, Gr::HI, Gr::LO>(x, gr.base_low, twi, p);
            if constexpr (NR == 1) {
#pragma unroll
                for (int j = 0; j < (1 << R); ++j) x[j] = Bfly<LAZY>::reduce(x[j], p);
            }
#pragma unroll
            for (int j = 0; j < (1 << R); ++j) s[gr.at(j)] = x[j];
        }
    }
    __syncthreads();
    if constexpr (NR > 1) {
        dit_rounds<LAZY, L2, kCols, TP, NR - 2, 1>(s, twi, p, tq);
        // Round 0: DIT then reduce to [0, p) for the CRT.
        using Gr = Group<L2, kCols, 0>;
        constexpr int R = Gr::R;
#pragma unroll 2
        for (int g = tq; g < Gr::G; g += TP) {
            const Gr gr(g);
            uint32_t x[1 << R];
#pragma unroll
            for (int j = 0; j < (1 << R); ++j) x[j] = s[gr.at(j)];
            dit_regs<LAZY, R, Gr::HI, Gr::LO>(x, gr.base_low, twi, p);
#pragma unroll
            for (int j = 0; j < (1 << R); ++j) s[gr.at(j)] = Bfly<LAZY>::reduce(x[j], p);
        }
        __syncthreads();
    }

    // CRT and chunk sums: row n2 of the tile is chunk (c0 + N1*n2)/8.
#pragma unroll 2
    for (uint32_t n2 = threadIdx.x; n2 < (1u << L2); n2 += T) {
        uint32_t w0[kCols], w1[kCols], w2[kCols];
        const uint32_t row = sidx<kCols>(n2, 0);
        const uint4* s0 = reinterpret_cast<const uint4*>(sm + row);
        const uint4* s1 = reinterpret_cast<const uint4*>(sm + TILE + row);
        const uint4* s2 = reinterpret_cast<const uint4*>(sm + 2 * TILE + row);
        uint32_t r0[kCols], r1[kCols], r2[kCols];
#pragma unroll
        for (int h = 0; h < kCols / 4; ++h) {
            uint4 u = s0[h], v = s1[h], t = s2[h];
            r0[4 * h] = u.x, r0[4 * h + 1] = u.y, r0[4 * h + 2] = u.z, r0[4 * h + 3] = u.w;
            r1[4 * h] = v.x, r1[4 * h + 1] = v.y, r1[4 * h + 2] = v.z, r1[4 * h + 3] = v.w;
            r2[4 * h] = t.x, r2[4 * h + 1] = t.y, r2[4 * h + 2] = t.z, r2[4 * h + 3] = t.w;
        }
#pragma unroll
        for (int i = 0; i < kCols; ++i) crt3(c, r0[i], r1[i], r2[i], w0[i], w1[i], w2[i]);
        // digit k = w0[k] + w1[k-1] + w2[k-2] + carry, k = 0..9
        uint32_t d[kCols + 2];
        uint64_t carry = 0;
#pragma unroll
        for (int k = 0; k < kCols + 2; ++k) {
            uint64_t s = carry;
            if (k < kCols) s += w0[k];
            if (k >= 1 && k - 1 < kCols) s += w1[k - 1];
            if (k >= 2 && k - 2 < kCols) s += w2[k - 2];
            d[k] = (uint32_t)s;
            carry = s >> 32;
        }
        const size_t chunk = (size_t)(c0 / kCols) + (size_t)(n1_len / kCols) * n2;
        ulonglong2* dst = reinterpret_cast<ulonglong2*>(pd.chunks + chunk * 4);
        dst[0] = make_ulonglong2(d[0] | ((uint64_t)d[1] << 32), d[2] | ((uint64_t)d[3] << 32));
        dst[1] = make_ulonglong2(d[4] | ((uint64_t)d[5] << 32), d[6] | ((uint64_t)d[7] << 32));
        pd.spill[chunk] = d[8] | ((uint64_t)d[9] << 32);
    }
}

template <int PS, int L2, int TP>
__global__ void __launch_bounds__(kNumPrimes * TP) k_inv_cols(const InvColsArgs a) {
    extern __shared__ __align__(16) uint32_t sm[];
    inv_cols_body<PS, L2, TP>(a, blockIdx.x, blockIdx.y, sm);
}

// ---- kernel 4: carry scan with decoupled look-back ----------------------------

constexpr uint32_t kSpinLimit = 1u << 22;  // bounded look-back wait, then error exit

struct CarryArgs {
    const ProductDesc* descs;  // chunks, spill, flags, out, out_cap per product
    ProductDesc one;
    uint32_t nchunks;  // real chunks per product; chunk nchunks is a virtual all-zero chunk
    uint32_t bpp;      // carry blocks per product
    int out_fmt;
    unsigned long long* ticket;
    uint64_t ticket_base;
    uint64_t epoch;
    uint32_t* err;
};

// Flag word: [63:4] epoch, [3:2] status (1 aggregate, 2 inclusive), [1] G/carry, [0] P.
__device__ __forceinline__ uint64_t make_flag(uint64_t epoch, uint32_t status, uint32_t g,
                                              uint32_t pbit) {
    return (epoch << 4) | ((uint64_t)status << 2) | ((uint64_t)g << 1) | pbit;
}

// Bounded wait for a look-back flag word of the current epoch: returns it, or
// 0 after `limit` polls with bit 0 of the error word set.  The only wait of
// the carry scan; the diagnostic k_wait_selftest runs it on its own.
__device__ __forceinline__ uint64_t wait_flag(const uint64_t* flag, uint64_t epoch, uint32_t limit,
                                              uint32_t* err) {
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> w(
        *reinterpret_cast<unsigned long long*>(const_cast<uint64_t*>(flag)));
    for (uint32_t spins = 0;; ++spins) {
        const uint64_t f = w.load(cuda::memory_order_acquire);
        if ((f >> 4) == epoch) return f;
        if (spins >= limit) {
            atomicOr(err, 1u);
            return 0;
        }
        __nanosleep(32);
    }
}

// Diagnostic: one thread waits on `flag` for `epoch` with the carry scan's
// wait; with a flag nothing sets it gives up after `limit` polls.
__global__ void k_wait_selftest(const uint64_t* flag, uint64_t epoch, uint32_t limit, uint32_t* err) {
    if (threadIdx.x == 0 && blockIdx.x == 0) wait_flag(flag, epoch, limit, err);
}

cudaError_t launch_wait_selftest(const uint64_t* flag, uint64_t epoch, uint32_t limit, uint32_t* err,
                                 cudaStream_t st) {
    k_wait_selftest<<<1, 32, 0, st>>>(flag, epoch, limit, err);
    return cudaGetLastError();
}

// Carry resolution over chunks of 8 coefficients.  Chunk c's final value is
// (D_c + spill_{c-1} + carry_c) mod 2^256 with carry_{c+1} = G_c | (P_c & carry_c),
// G_c = "D_c + spill_{c-1} >= 2^256", P_c = "D_c + spill_{c-1} == 2^256 - 1".
// A block covers kCarryThreads * kCarryPer consecutive chunks; warp w of the
// block owns 32 * kCarryPer of them as kCarryPer segments of 32, lane l
// holding chunk (segment base + l), so every load and store of a segment is
// one contiguous run over the warp.  All loads are issued before any carry
// logic (one memory round trip).  Carries inside a segment come from one
// 64-bit add of the (G, P) ballots; segments are chained inside the warp,
// warps by a fold in shared memory, and blocks by a decoupled look-back in
// ticket order.
// Block `bid` of one product's carry scan over `nchunks` chunks, writing the
// output in `out_fmt`; blocks of the same product must hold increasing
// tickets of one launch (their look-back waits only on earlier blocks).
template <int TH, int PER>
__device__ __forceinline__ void carry_block(const ProductDesc& pd, uint32_t bid, uint32_t nchunks, int out_fmt,
                                            uint64_t epoch, uint32_t* err) {
    constexpr uint32_t CPB = (uint32_t)(TH * PER);  // chunks per block
    __shared__ uint32_t s_cin, s_win_g, s_win_p;
    __shared__ uint32_t s_wg[TH / 32], s_wp[TH / 32];
    const uint64_t* chunks = pd.chunks;
    const uint64_t* spill = pd.spill;
    uint64_t* flags = pd.flags;
    const size_t out_cap = pd.out_cap;
    const uint32_t ntot = nchunks + 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t wbase = (bid * TH + (uint32_t)warp * 32) * PER;

    // every load first: chunk words and the spill of the chunk before
    uint64_t S[PER][4], sp[PER];
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        const uint32_t cc = wbase + (uint32_t)i * 32 + lane;
        if (cc < nchunks) {
            const ulonglong2* src = reinterpret_cast<const ulonglong2*>(chunks + (size_t)cc * 4);
            const ulonglong2 u = src[0], v = src[1];
            S[i][0] = u.x, S[i][1] = u.y, S[i][2] = v.x, S[i][3] = v.y;
        } else {
            S[i][0] = S[i][1] = S[i][2] = S[i][3] = 0;
        }
        sp[i] = (cc >= 1 && cc - 1 < nchunks) ? spill[cc - 1] : 0;
    }
    // Warp 0 also reads the 32 chunks below the block (all real chunks: the
    // block starts at or below the last one) and records their (G, P): the
    // carry into the block is the G of the highest of them that does not
    // propagate, found without waiting on any other block.
    if (warp == 0) {
        const int64_t j = (int64_t)bid * CPB - 32 + lane;
        uint32_t g = 0, pbit = 0;  // below chunk 0: no carry, nothing propagates
        if (j >= 0) {
            const ulonglong2* src = reinterpret_cast<const ulonglong2*>(chunks + (size_t)j * 4);
            const ulonglong2 u = src[0], v = src[1];
            const uint64_t s0 = j >= 1 ? spill[j - 1] : 0;
            const uint64_t t0 = u.x + s0;
            uint32_t cy = t0 < s0;
            const uint64_t t1 = u.y + cy;
            cy = cy & (t1 == 0);
            const uint64_t t2 = v.x + cy;
            cy = cy & (t2 == 0);
            const uint64_t t3 = v.y + cy;
            cy = cy & (t3 == 0);
            g = cy;
            pbit = (!cy) && ((t0 & t1 & t2 & t3) == ~0ull);
        }
        const uint32_t wg = __ballot_sync(0xffffffffu, g), wp = __ballot_sync(0xffffffffu, pbit);
        if (lane == 0) {
            s_win_g = wg;
            s_win_p = wp;
        }
    }
    // per-chunk (G, P) and per-segment ballots
    uint32_t gm[PER], bm[PER];
    uint32_t G = 0, P = 1;  // warp aggregate over its segments
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        const uint32_t cc = wbase + (uint32_t)i * 32 + lane;
        uint32_t g = 0, pbit = 1;  // chunks past the end pass carries through untouched
        if (cc < ntot) {
            uint64_t t = S[i][0] + sp[i];
            uint32_t cy = t < sp[i];
            S[i][0] = t;
#pragma unroll
            for (int k = 1; k < 4; ++k) {
                t = S[i][k] + cy;
                cy = cy & (t == 0);
                S[i][k] = t;
            }
            g = cy;
            pbit = (!cy) && ((S[i][0] & S[i][1] & S[i][2] & S[i][3]) == ~0ull);
        }
        const uint32_t gmi = __ballot_sync(0xffffffffu, g);
        const uint32_t pmi = __ballot_sync(0xffffffffu, pbit);
        gm[i] = gmi;
        bm[i] = gmi | pmi;
        const uint32_t segG = (uint32_t)((((uint64_t)gmi + bm[i]) >> 32) & 1u);
        G = segG | ((pmi == 0xffffffffu) & G);
        P = P & (pmi == 0xffffffffu);
    }
    if (lane == 0) {
        s_wg[warp] = G;
        s_wp[warp] = P;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t bG = 0, bP = 1;
        for (int w = 0; w < TH / 32; ++w) {
            bG = s_wg[w] | (s_wp[w] & bG);
            bP = bP & s_wp[w];
        }
        uint32_t cin = 0;
        cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> self(
            *reinterpret_cast<unsigned long long*>(flags + bid));
        const uint32_t stop = ~s_win_p;  // window chunks that do not propagate a carry
        if (bid == 0) {
            self.store(make_flag(epoch, 2, bG, 0), cuda::memory_order_release);
        } else if (stop) {
            cin = (s_win_g >> (31 - __clz(stop))) & 1u;  // the highest one's carry out
            self.store(make_flag(epoch, 2, bG | (bP & cin), 0), cuda::memory_order_release);
        } else {  // 32 propagating chunks: the decoupled look-back on the blocks' flags
            self.store(make_flag(epoch, 1, bG, bP), cuda::memory_order_release);
            int k = (int)bid - 1;
            while (true) {
                const uint64_t f = wait_flag(flags + k, epoch, kSpinLimit, err);
                if (f == 0) break;  // gave up: error recorded, carry taken as 0
                const uint32_t st = (uint32_t)(f >> 2) & 3u, fg = (uint32_t)(f >> 1) & 1u,
                               fp = (uint32_t)f & 1u;
                if (st == 2) {
                    cin = fg;
                    break;
                }
                if (fg) {
                    cin = 1;
                    break;
                }
                if (!fp) {
                    cin = 0;
                    break;
                }
                --k;  // predecessor propagates: look further back (block 0 is inclusive)
            }
            self.store(make_flag(epoch, 2, bG | (bP & cin), 0), cuda::memory_order_release);
        }
        s_cin = cin;
    }
    __syncthreads();
    uint32_t cw = s_cin;  // carry into this warp's first segment
    for (int w = 0; w < warp; ++w) cw = s_wg[w] | (s_wp[w] & cw);
    uint32_t cout[PER];  // carry out of each of this lane's chunks
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        const uint64_t sum = (uint64_t)gm[i] + bm[i] + cw;
        const uint32_t carries = (uint32_t)sum ^ gm[i] ^ bm[i];
        const uint32_t cin = (carries >> lane) & 1u;
        // carry out of lane l is the carry into lane l+1 (bit 32 for lane 31)
        cout[i] = lane == 31 ? (uint32_t)(sum >> 32) & 1u : (carries >> (lane + 1)) & 1u;
        cw = (uint32_t)(sum >> 32) & 1u;
        uint32_t cy = cin;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint64_t t = S[i][k] + cy;
            cy = cy & (t == 0);
            S[i][k] = t;
        }
    }
    if (out_fmt == kFmtLimb64) {
        uint64_t* o = static_cast<uint64_t*>(pd.out);
        const bool vec = (reinterpret_cast<uintptr_t>(o) & 15u) == 0;  // 16-byte stores when aligned
#pragma unroll
        for (int i = 0; i < PER; ++i) {
            const uint32_t cc = wbase + (uint32_t)i * 32 + lane;
            if (cc >= ntot) continue;
            const size_t base = (size_t)cc * 4;
            if (base + 4 <= out_cap && vec) {
                ulonglong2* d = reinterpret_cast<ulonglong2*>(o + base);
                d[0] = make_ulonglong2(S[i][0], S[i][1]);
                d[1] = make_ulonglong2(S[i][2], S[i][3]);
            } else if (base + 4 <= out_cap) {
#pragma unroll
                for (int k = 0; k < 4; ++k) o[base + k] = S[i][k];
            } else {
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (base + k < out_cap) o[base + k] = S[i][k];
            }
        }
    } else {
        // 28-bit digits starting in each chunk; the last one may reach into
        // chunk cc+1, whose final low limb is its raw limb plus this chunk's
        // spill plus the carry out of this chunk (mod 2^64 suffices).
        uint32_t* o = static_cast<uint32_t*>(pd.out);
        const uint64_t mask = (1u << 28) - 1u;
#pragma unroll
        for (int i = 0; i < PER; ++i) {
            const uint32_t cc = wbase + (uint32_t)i * 32 + lane;
            if (cc >= ntot) continue;
            uint64_t nl = (cc + 1 < nchunks) ? chunks[(size_t)(cc + 1) * 4] : 0;
            nl += (cc < nchunks ? spill[cc] : 0) + cout[i];
            const uint64_t bit0 = (uint64_t)cc * 256;
            uint64_t k = (bit0 + 27) / 28;
            const uint64_t kend = min((bit0 + 256 + 27) / 28, (uint64_t)out_cap);
            const uint32_t off0 = (uint32_t)(k * 28 - bit0);  // < 28
            uint64_t cur = S[i][0] >> off0;
            int have = 64 - (int)off0;
#pragma unroll
            for (int w = 1; w <= 4; ++w) {
                const uint64_t nxtw = w < 4 ? S[i][w] : nl;
                while (have >= 28) {
                    if (k < kend) o[k] = (uint32_t)(cur & mask);
                    ++k;
                    cur >>= 28;
                    have -= 28;
                }
                if (k < kend) o[k] = (uint32_t)((cur | (nxtw << have)) & mask);
                ++k;
                cur = nxtw >> (28 - have);
                have = 36 + have;
            }
        }
    }
}

template <int TH, int PER>
__global__ void __launch_bounds__(TH) k_carry(const CarryArgs a) {
    __shared__ uint32_t s_bid;
    if (threadIdx.x == 0) s_bid = (uint32_t)(atomicAdd(a.ticket, 1ull) - a.ticket_base);
    __syncthreads();
    pdl_wait();
    pdl_trigger();
    // A ticket outside this launch means the host's ticket base and the
    // counter disagree (an earlier launch that never ran): report, touch nothing.
    if (s_bid >= gridDim.x) {
        if (threadIdx.x == 0) atomicOr(a.err, 2u);
        return;
    }
    // tickets enumerate (product, block) in order, so a block's predecessor
    // within its product always holds a smaller ticket
    carry_block<TH, PER>(product(a.descs, a.one, s_bid / a.bpp), s_bid % a.bpp, a.nchunks, a.out_fmt, a.epoch,
                         a.err);
}

// Before the carry scan of a spectral sum that lands in a window of the
// result already holding earlier sums: chunk c's value (4 limbs + 2^256 *
// spill[c]) becomes twice itself when `twice` (a square's off-diagonal
// pairs), plus limbs 4c..4c+3 of the window; the top limb past the chunks
// (the carry scan's extra chunk, which is spill[nchunks-1]) takes window
// limb 4 nchunks.  A chunk's overflow above 256 bits goes into its spill, so
// the scan still sees chunk + spill below 2^257.  Spills stay below 2^61:
// the coefficients are below 2^91, a chunk's top one shifted by 224 bits, and
// the window's top limb is 0 before its first sum and after it below the
// number of block products carried there.
struct ChunkMerge {
    const uint64_t* add;  // window limbs to add, or nullptr
    uint64_t nadd;
    int twice;
    uint64_t* chunks;  // the product's chunk sums and spills (set by the launcher)
    uint64_t* spill;
    uint32_t nchunks;
};

__global__ void __launch_bounds__(256) k_chunks_merge(const ChunkMerge m) {
    pdl_wait();
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nchunks = m.nchunks;
    if (c < nchunks) {
        ulonglong2* p = reinterpret_cast<ulonglong2*>(m.chunks + (size_t)c * 4);
        const ulonglong2 u = p[0], v = p[1];
        uint64_t s[4] = {u.x, u.y, v.x, v.y};
        uint64_t sp = m.spill[c];
        if (m.twice) {
            sp = (sp << 1) | (s[3] >> 63);
            s[3] = (s[3] << 1) | (s[2] >> 63);
            s[2] = (s[2] << 1) | (s[1] >> 63);
            s[1] = (s[1] << 1) | (s[0] >> 63);
            s[0] <<= 1;
        }
        const uint64_t base = (uint64_t)c * 4;
        uint64_t cy = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint64_t w = base + k < m.nadd ? m.add[base + k] : 0ull;
            const uint64_t t = s[k] + w;
            const uint64_t r = t + cy;
            cy = (uint64_t)(t < w) | (uint64_t)(r < t);
            s[k] = r;
        }
        sp += cy;
        if (c == nchunks - 1 && m.nadd > base + 4) sp += m.add[base + 4];
        p[0] = make_ulonglong2(s[0], s[1]);
        p[1] = make_ulonglong2(s[2], s[3]);
        m.spill[c] = sp;
    }
    pdl_trigger();
}

// ---- host launchers -------------------------------------------------------------

// Column length per transform length, as set by the tuner (0 = default
// split): one table for single products (latency) and one for the NTT
// classes of batch plans and product-tree levels (throughput).
static int g_split[kMaxLogN + 1] = {};
static int g_batch_split[kMaxLogN + 1] = {};

static int set_split_in(int* table, int log_n, int log_n2) {
    if (log_n < 5 || log_n > kMaxLogN) return -1;
    if (log_n2 != 0) {
        const int l1 = log_n - log_n2;
        if (log_n2 < 2 || log_n2 > 11 || l1 < 3 || l1 > 15) return -1;
    }
    table[log_n] = log_n2;
    return 0;
}

int set_split(int log_n, int log_n2) { return set_split_in(g_split, log_n, log_n2); }
int set_batch_split(int log_n, int log_n2) { return set_split_in(g_batch_split, log_n, log_n2); }

TransformShape builtin_shape(int log_n) {
    TransformShape s;
    s.log_n = log_n;
    int l2 = (log_n - 1) / 2;
    if (l2 > 11) l2 = 11;
    if (l2 < 2) l2 = 2;
    s.log_n2 = l2;
    s.log_n1 = log_n - l2;
    return s;
}

static TransformShape shape_from(const int* table, int log_n) {
    TransformShape s = builtin_shape(log_n);
    if (log_n >= 0 && log_n <= kMaxLogN && table[log_n]) {
        s.log_n2 = table[log_n];
        s.log_n1 = log_n - s.log_n2;
    }
    return s;
}

TransformShape choose_shape(int log_n) { return shape_from(g_split, log_n); }
TransformShape choose_shape_batch(int log_n) { return shape_from(g_batch_split, log_n); }

static bool shape_ok(const TransformShape& s, bool square) {
    if (s.log_n < 5 || s.log_n > kMaxLogN) return false;
    if (s.log_n2 < 2 || s.log_n2 > 11) return false;
    if (s.log_n1 < 3 || s.log_n1 > 15) return false;
    // Rows of 2^15 points are built for the strict prime set only (transforms
    // above 2^23 points); non-square products use the one-buffer row pass.
    if (s.log_n1 == 15 && prime_set_for(s.log_n) == 0) return false;
    (void)square;
    return true;
}

bool shape_supported(int log_n, bool square) { return shape_ok(choose_shape(log_n), square); }
bool shape_supported_batch(int log_n, bool square) { return shape_ok(choose_shape_batch(log_n), square); }

size_t smem_fwd_cols(int l2, int cols) { return ((size_t)cols * 4 << l2) + cols * 17 * sizeof(uint2); }
size_t smem_mid_rows(int l1, bool square) {
    return (square || l1 >= 15 ? 1 : 2) * ((size_t)4 << l1) + 16 * sizeof(uint2);
}
size_t smem_inv_cols(int l2) { return (size_t)kNumPrimes * kCols * 4 << l2; }

static constexpr int mid_threads(int l1) { return l1 >= 12 ? 256 : (l1 >= 9 ? (1 << (l1 - 4)) : 32); }


template <int PS, int L2>
static cudaError_t launch_outer(const FwdColsArgs* f, const InvColsArgs* inv, uint32_t tiles,
                                int count, cudaStream_t st) {
#ifndef BGPU_INV_TP
#define BGPU_INV_TP 128
#endif
    constexpr int TP = BGPU_INV_TP;
    if (f) {
        // `tiles` counts 8-column tiles; the forward pass's tiles are kFwdCols wide
        auto k = k_fwd_cols<PS, L2, kFwdThreads>;
        const size_t sm = smem_fwd_cols(L2, kFwdCols);
        allow_smem(k, sm);
        return launch_k(k, dim3(tiles * (kCols / kFwdCols), kNumPrimes, f->nops * count), dim3(kFwdThreads), sm,
                        st, *f);
    }
    auto k = k_inv_cols<PS, L2, TP>;
    const size_t sm = smem_inv_cols(L2);
    allow_smem(k, sm);
    return launch_k(k, dim3(tiles, count), dim3(kNumPrimes * TP), sm, st, *inv);
}

template <int PS>
static cudaError_t dispatch_outer(int l2, const FwdColsArgs* f, const InvColsArgs* inv,
                                  uint32_t tiles, int count, cudaStream_t st) {
    switch (l2) {
        case 2: return launch_outer<PS, 2>(f, inv, tiles, count, st);
        case 3: return launch_outer<PS, 3>(f, inv, tiles, count, st);
        case 4: return launch_outer<PS, 4>(f, inv, tiles, count, st);
        case 5: return launch_outer<PS, 5>(f, inv, tiles, count, st);
        case 6: return launch_outer<PS, 6>(f, inv, tiles, count, st);
        case 7: return launch_outer<PS, 7>(f, inv, tiles, count, st);
        case 8: return launch_outer<PS, 8>(f, inv, tiles, count, st);
        case 9: return launch_outer<PS, 9>(f, inv, tiles, count, st);
        case 10: return launch_outer<PS, 10>(f, inv, tiles, count, st);
        case 11: return launch_outer<PS, 11>(f, inv, tiles, count, st);
        default: return cudaErrorInvalidValue;
    }
}

template <int PS, int L1>
static cudaError_t launch_mid(const MidRowsArgs& m, bool square, uint32_t rows, int count,
                              cudaStream_t st) {
    constexpr int T = mid_threads(L1);
    const size_t sm = smem_mid_rows(L1, square);
    const dim3 grid(rows, kNumPrimes * count);
    if (square) {
        auto k = k_mid_rows<PS, L1, T, true>;
        allow_smem(k, sm);
        return launch_k(k, grid, dim3(T), sm, st, m);
    }
    auto k = k_mid_rows<PS, L1, T, false>;
    allow_smem(k, sm);
    return launch_k(k, grid, dim3(T), sm, st, m);
}

template <int PS>
static cudaError_t dispatch_mid(int l1, const MidRowsArgs& m, bool square, uint32_t rows, int count,
                                cudaStream_t st) {
    switch (l1) {
        case 3: return launch_mid<PS, 3>(m, square, rows, count, st);
        case 4: return launch_mid<PS, 4>(m, square, rows, count, st);
        case 5: return launch_mid<PS, 5>(m, square, rows, count, st);
        case 6: return launch_mid<PS, 6>(m, square, rows, count, st);
        case 7: return launch_mid<PS, 7>(m, square, rows, count, st);
        case 8: return launch_mid<PS, 8>(m, square, rows, count, st);
        case 9: return launch_mid<PS, 9>(m, square, rows, count, st);
        case 10: return launch_mid<PS, 10>(m, square, rows, count, st);
        case 11: return launch_mid<PS, 11>(m, square, rows, count, st);
        case 12: return launch_mid<PS, 12>(m, square, rows, count, st);
        case 13: return launch_mid<PS, 13>(m, square, rows, count, st);
        case 14: return launch_mid<PS, 14>(m, square, rows, count, st);
        case 15:
            if constexpr (PS == 1) return launch_mid<PS, 15>(m, square, rows, count, st);
            return cudaErrorInvalidValue;
        default: return cudaErrorInvalidValue;
    }
}

// Row lengths of the spectral row passes: several rounds (2^5 points and up);
// the lazy set's transforms (up to 2^23 points) have rows of at most 2^14,
// the strict set's (2^24 to 2^26 points, columns of at most 2^11) at least 2^13.
static bool spec_rows_built(int ps, int l1) { return ps == 0 ? (l1 >= 5 && l1 <= 14) : (l1 >= 13 && l1 <= 15); }

// Threads of the spectral row passes: rows of 2^13 points and more fill one
// or two CTAs per SM (their shared rows take 32-128 KB), so these run 512
// threads, twice the row pass's, for more global loads in flight.
static constexpr int spec_threads(int l1) { return l1 >= 13 ? 512 : mid_threads(l1); }

template <int PS, int L1, int NT>
static cudaError_t launch_spec_mac(const SpecArgs& s, uint32_t rows, cudaStream_t st) {
    constexpr int T = spec_threads(L1);
    auto k = k_rows_mac<PS, L1, T, NT>;
    const size_t sm = ((size_t)4 << L1) + 16 * sizeof(uint2);
    allow_smem(k, sm);
    return launch_k(k, dim3(rows, kNumPrimes), dim3(T), sm, st, s);
}

template <int PS, int L1>
static cudaError_t launch_spec_rows(const SpecArgs& s, bool mac, uint32_t rows, cudaStream_t st) {
    constexpr int T = spec_threads(L1);
    const dim3 grid(rows, kNumPrimes);
    if (mac) {
        // the strict set's transforms are the large blocks, whose sums hold
        // one or two products; other counts and the small blocks' sums take
        // the general loop
        if constexpr (PS == 1) {
            if (s.nterms == 1) return launch_spec_mac<PS, L1, 1>(s, rows, st);
            if (s.nterms == 2) return launch_spec_mac<PS, L1, 2>(s, rows, st);
        }
        return launch_spec_mac<PS, L1, 0>(s, rows, st);
    }
    auto k = k_rows_dif<PS, L1, T>;
    const size_t sm = (size_t)4 << L1;
    allow_smem(k, sm);
    return launch_k(k, grid, dim3(T), sm, st, s);
}

template <int PS>
static cudaError_t dispatch_spec_rows(int l1, const SpecArgs& s, bool mac, uint32_t rows, cudaStream_t st) {
    if constexpr (PS == 0) {
        switch (l1) {
            case 5: return launch_spec_rows<0, 5>(s, mac, rows, st);
            case 6: return launch_spec_rows<0, 6>(s, mac, rows, st);
            case 7: return launch_spec_rows<0, 7>(s, mac, rows, st);
            case 8: return launch_spec_rows<0, 8>(s, mac, rows, st);
            case 9: return launch_spec_rows<0, 9>(s, mac, rows, st);
            case 10: return launch_spec_rows<0, 10>(s, mac, rows, st);
            case 11: return launch_spec_rows<0, 11>(s, mac, rows, st);
            case 12: return launch_spec_rows<0, 12>(s, mac, rows, st);
            case 13: return launch_spec_rows<0, 13>(s, mac, rows, st);
            case 14: return launch_spec_rows<0, 14>(s, mac, rows, st);
            default: return cudaErrorInvalidValue;
        }
    } else {
        switch (l1) {
            case 13: return launch_spec_rows<1, 13>(s, mac, rows, st);
            case 14: return launch_spec_rows<1, 14>(s, mac, rows, st);
            case 15: return launch_spec_rows<1, 15>(s, mac, rows, st);
            default: return cudaErrorInvalidValue;
        }
    }
}

uint32_t carry_blocks(uint32_t nchunks) {
    return (nchunks + 1 + kCarryChunksPerBlock - 1) / kCarryChunksPerBlock;
}

uint32_t carry_blocks_narrow(uint32_t nchunks) {
    constexpr uint32_t cpb = (uint32_t)(kCarryNarrowThreads * kCarryNarrowPer);
    return (nchunks + 1 + cpb - 1) / cpb;
}

static uint32_t mont_of(uint64_t v, uint32_t p) { return (uint32_t)((v % p << 32) % p); }

// The row pass's scale per prime: the pointwise Montgomery product leaves a
// factor 2^-32; the scale N^-1 * 2^32 (mod p) cancels it and applies the
// inverse's 1/N (Montgomery pairs).
static void set_scale(const NttConsts& c, int log_n, uint32_t* w, uint32_t* wp) {
    for (int q = 0; q < kNumPrimes; ++q) {
        const uint32_t p = c.pr[q].p;
        uint64_t ninv = 1, base = (p + 1) / 2;  // 2^-1 mod p
        for (int i = 0; i < log_n; ++i) ninv = ninv * base % p;
        const uint64_t r = ((uint64_t)1 << 32) % p;
        const uint64_t v = ninv * r % p;
        w[q] = mont_of(v, p);
        wp[q] = w[q] * c.pr[q].pinv;
    }
}

// The four launches of `count` products (descs on the device, or `one`).
static cudaError_t launch_inverse_carry(int slot, int ps, const ProductDesc* descs, const ProductDesc& one,
                                        int count, const TransformShape& sh, int out_fmt,
                                        const CarryLaunch& cl, cudaStream_t st, cudaEvent_t* ev,
                                        const ChunkMerge* merge = nullptr);

static cudaError_t launch_ntt_core(int slot, const NttConsts& c, const ProductDesc* descs,
                                   const ProductDesc& one, int count, bool square,
                                   const TransformShape& sh, int out_fmt, const CarryLaunch& cl,
                                   cudaStream_t st, cudaEvent_t* ev) {
    const int log_n = sh.log_n;
    if (!shape_ok(sh, square) || log_n > c.log_max || count < 1) return cudaErrorInvalidValue;
    const int ps = c.log_max == kPrimeSets[0].log_max ? 0 : 1;
    const uint32_t tiles = (1u << sh.log_n1) / kCols;
    if (ev) cudaEventRecord(ev[0], st);

    FwdColsArgs f{};
    f.descs = descs;
    f.one = one;
    f.nops = square ? 1 : 2;
    f.log_n = log_n;
    f.log_n1 = sh.log_n1;
    f.slot = slot;
    f.overlap = cl.overlap_prev && count == 1 ? 1 : 0;
    cudaError_t e = ps == 0 ? dispatch_outer<0>(sh.log_n2, &f, nullptr, tiles, count, st)
                            : dispatch_outer<1>(sh.log_n2, &f, nullptr, tiles, count, st);
    if (e != cudaSuccess) return e;
    if (ev) cudaEventRecord(ev[1], st);

    MidRowsArgs m{};
    m.descs = descs;
    m.one = one;
    m.log_n = log_n;
    m.log_n2 = sh.log_n2;
    m.slot = slot;
    set_scale(c, log_n, m.scale_w, m.scale_wp);
    e = ps == 0 ? dispatch_mid<0>(sh.log_n1, m, square, 1u << sh.log_n2, count, st)
                : dispatch_mid<1>(sh.log_n1, m, square, 1u << sh.log_n2, count, st);
    if (e != cudaSuccess) return e;
    if (ev) cudaEventRecord(ev[2], st);
    return launch_inverse_carry(slot, ps, descs, one, count, sh, out_fmt, cl, st, ev);
}

// The inverse column pass (with CRT and chunk sums) and the carry scan of
// `count` products whose row pass has run; `merge` (one product only) runs
// k_chunks_merge between them.
static cudaError_t launch_inverse_carry(int slot, int ps, const ProductDesc* descs, const ProductDesc& one,
                                        int count, const TransformShape& sh, int out_fmt,
                                        const CarryLaunch& cl, cudaStream_t st, cudaEvent_t* ev,
                                        const ChunkMerge* merge) {
    const int log_n = sh.log_n;
    const size_t nn = (size_t)1 << log_n;
    const uint32_t tiles = (1u << sh.log_n1) / kCols;
    InvColsArgs iv{};
    iv.descs = descs;
    iv.one = one;
    iv.log_n = log_n;
    iv.log_n1 = sh.log_n1;
    iv.slot = slot;
    iv.err = cl.err;
    cudaError_t e = ps == 0 ? dispatch_outer<0>(sh.log_n2, nullptr, &iv, tiles, count, st)
                : dispatch_outer<1>(sh.log_n2, nullptr, &iv, tiles, count, st);
    if (e != cudaSuccess) return e;
    if (ev) cudaEventRecord(ev[3], st);
    if (merge) {
        ChunkMerge mg = *merge;
        mg.chunks = one.chunks;
        mg.spill = one.spill;
        mg.nchunks = (uint32_t)(nn / kCols);
        e = launch_k(k_chunks_merge, dim3((mg.nchunks + 255) / 256), dim3(256), 0, st, mg);
        if (e != cudaSuccess) return e;
    }

    CarryArgs ca{};
    ca.descs = descs;
    ca.one = one;
    ca.nchunks = (uint32_t)(nn / kCols);
    ca.out_fmt = out_fmt;
    ca.ticket = cl.ticket;
    ca.ticket_base = cl.ticket_base;
    ca.epoch = cl.epoch;
    ca.err = cl.err;
    if (cl.narrow && count == 1) {
        ca.bpp = carry_blocks_narrow(ca.nchunks);
        e = launch_k(k_carry<kCarryNarrowThreads, kCarryNarrowPer>, dim3(ca.bpp), dim3(kCarryNarrowThreads), 0, st,
                     ca);
    } else {
        ca.bpp = carry_blocks(ca.nchunks);
        e = launch_k(k_carry<kCarryThreads, kCarryPer>, dim3(ca.bpp * count), dim3(kCarryThreads), 0, st, ca);
    }
    if (ev) cudaEventRecord(ev[4], st);
    return e;
}

cudaError_t launch_ntt_product(int slot, const NttConsts& c, const OperandDesc& a,
                               const OperandDesc& b, bool square, int log_n,
                               const ProductScratch& s, void* out, int out_fmt, size_t out_cap,
                               const CarryLaunch& cl, cudaStream_t st, cudaEvent_t* ev,
                               const TransformShape* shape) {
    ProductDesc one{};
    one.op[0] = a;
    one.op[1] = square ? a : b;
    one.y = s.y;
    one.chunks = s.chunks;
    one.spill = s.spill;
    one.flags = s.flags;
    one.out = out;
    one.out_cap = out_cap;
    CarryLaunch c2 = cl;
    c2.ticket = s.ticket;
    c2.err = s.err;
    return launch_ntt_core(slot, c, nullptr, one, 1, square, shape ? *shape : choose_shape(log_n),
                           out_fmt, c2, st, ev);
}

cudaError_t launch_ntt_batch(int slot, const NttConsts& c, const ProductDesc* descs, int count,
                             bool square, int log_n, int out_fmt, const CarryLaunch& cl,
                             cudaStream_t st) {
    // Grid y/z limits (65535) cap the products of one launch; larger batches
    // go in pieces, each piece's carry scan continuing the ticket sequence.
    constexpr int kPiece = 16384;
    const uint32_t bpp = carry_blocks((uint32_t)(((size_t)1 << log_n) / kCols));
    for (int done = 0; done < count; done += kPiece) {
        const int n = count - done < kPiece ? count - done : kPiece;
        CarryLaunch piece = cl;
        piece.ticket_base = cl.ticket_base + (uint64_t)done * bpp;
        const cudaError_t e = launch_ntt_core(slot, c, descs + done, ProductDesc{}, n, square,
                                              choose_shape_batch(log_n), out_fmt, piece, st, nullptr);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

bool spectral_supported(int log_n) {
    const TransformShape sh = choose_shape(log_n);
    return shape_ok(sh, false) && spec_rows_built(prime_set_for(log_n), sh.log_n1);
}

cudaError_t launch_ntt_spectrum(int slot, const NttConsts& c, const OperandDesc& a, int log_n, uint32_t* spec,
                                cudaStream_t st) {
    const TransformShape sh = choose_shape(log_n);
    const int ps = c.log_max == kPrimeSets[0].log_max ? 0 : 1;
    if (!spectral_supported(log_n) || log_n > c.log_max || ps != prime_set_for(log_n))
        return cudaErrorInvalidValue;
    ProductDesc one{};
    one.op[0] = one.op[1] = a;
    one.y = spec;
    FwdColsArgs f{};
    f.one = one;
    f.nops = 1;
    f.log_n = log_n;
    f.log_n1 = sh.log_n1;
    f.slot = slot;
    const uint32_t tiles = (1u << sh.log_n1) / kCols;
    cudaError_t e = ps == 0 ? dispatch_outer<0>(sh.log_n2, &f, nullptr, tiles, 1, st)
                            : dispatch_outer<1>(sh.log_n2, &f, nullptr, tiles, 1, st);
    if (e != cudaSuccess) return e;
    SpecArgs s{};
    s.y = spec;
    s.log_n = log_n;
    s.log_n2 = sh.log_n2;
    s.slot = slot;
    return ps == 0 ? dispatch_spec_rows<0>(sh.log_n1, s, false, 1u << sh.log_n2, st)
                   : dispatch_spec_rows<1>(sh.log_n1, s, false, 1u << sh.log_n2, st);
}

cudaError_t launch_ntt_spectral_sum(int slot, const NttConsts& c, const uint32_t* const* sa,
                                    const uint32_t* const* sb, int nterms, bool twice, int log_n,
                                    const ProductScratch& scr, uint64_t* out, size_t out_cap,
                                    const uint64_t* add, size_t nadd, const CarryLaunch& cl,
                                    cudaStream_t st) {
    const TransformShape sh = choose_shape(log_n);
    const int ps = c.log_max == kPrimeSets[0].log_max ? 0 : 1;
    if (!spectral_supported(log_n) || log_n > c.log_max || ps != prime_set_for(log_n) || nterms < 1 ||
        nterms > kMaxSpecTerms)
        return cudaErrorInvalidValue;
    SpecArgs s{};
    for (int t = 0; t < nterms; ++t) {
        s.sa[t] = sa[t];
        s.sb[t] = sb[t];
    }
    s.nterms = nterms;
    s.y = scr.y;
    s.log_n = log_n;
    s.log_n2 = sh.log_n2;
    s.slot = slot;
    set_scale(c, log_n, s.scale_w, s.scale_wp);
    cudaError_t e = ps == 0 ? dispatch_spec_rows<0>(sh.log_n1, s, true, 1u << sh.log_n2, st)
                            : dispatch_spec_rows<1>(sh.log_n1, s, true, 1u << sh.log_n2, st);
    if (e != cudaSuccess) return e;
    ProductDesc one{};
    one.y = scr.y;
    one.chunks = scr.chunks;
    one.spill = scr.spill;
    one.flags = scr.flags;
    one.out = out;
    one.out_cap = out_cap;
    CarryLaunch c2 = cl;
    c2.ticket = scr.ticket;
    c2.err = scr.err;
    const ChunkMerge merge{add, add ? (uint64_t)nadd : 0ull, twice ? 1 : 0, nullptr, nullptr, 0};
    return launch_inverse_carry(slot, ps, nullptr, one, 1, sh, kFmtLimb64, c2, st, nullptr,
                                (add || twice) ? &merge : nullptr);
}

cudaError_t launch_carry(const uint64_t* chunks, const uint64_t* spill, uint32_t nchunks, void* out,
                         int out_fmt, size_t out_cap, const ProductScratch& s, const CarryLaunch& cl,
                         cudaStream_t st) {
    CarryArgs ca{};
    ca.one.chunks = const_cast<uint64_t*>(chunks);
    ca.one.spill = const_cast<uint64_t*>(spill);
    ca.one.flags = s.flags;
    ca.one.out = out;
    ca.one.out_cap = out_cap;
    ca.nchunks = nchunks;
    ca.bpp = carry_blocks(nchunks);
    ca.out_fmt = out_fmt;
    ca.ticket = s.ticket;
    ca.ticket_base = cl.ticket_base;
    ca.epoch = cl.epoch;
    ca.err = s.err;
    return launch_k(k_carry<kCarryThreads, kCarryPer>, dim3(ca.bpp), dim3(kCarryThreads), 0, st, ca);
}

// ---- mixed-length batches: one launch per pass for every class -------------
//
// A batch of products of several transform lengths runs as four launches in
// all, one per pass, instead of four per length: each CTA finds its class
// (the classes' CTA ranges are consecutive, their first CTAs kept in the
// launch parameters) and runs that class's pass body with block coordinates
// computed from its place in the range.  The row pass packs 128 / T rows of T
// threads into one 128-thread CTA.  The carry scan takes one ticket sequence
// over all classes; a product's blocks hold consecutive tickets.  The small
// products of the batch ride along as CTAs of their own after those of the
// row pass (schoolbook, 128 threads) and the inverse pass (Karatsuba, 384
// threads), filling the passes' last waves,
// with their shared memory carved from the launch's dynamic buffer; they wait
// on nothing.  Classes qualify when they use the lazy prime set, column tiles
// of at most 2^9 rows and rows of at most 2^9 points (mixed_class_ok), which
// keeps each launch's registers near the per-length kernels'.

constexpr int kMixedMidThreads = 128;
// Register budgets of the mixed launches (each holds every length's body):
// 7 forward CTAs of 256 threads per SM (32 registers, some spilled; measured
// on the 4096-product batch: 10.71 ms against 10.88 ms at 40 registers and 6
// CTAs), 7 row CTAs of 128 threads (72 registers, what a 2^9-point row takes
// on its own; 6 CTAs at 80 registers measured 10.87 ms).
#ifndef BGPU_MIXED_FWD_MINB
#define BGPU_MIXED_FWD_MINB 7
#endif
#ifndef BGPU_MIXED_MID_MINB
#define BGPU_MIXED_MID_MINB 7
#endif

__device__ __forceinline__ int mixed_class(const MixedArgs& m, int pass, uint32_t b) {
    int c = 0;
    while (c + 1 < m.nclasses && m.begin[pass][c + 1] <= b) ++c;
    return c;
}

__global__ void __launch_bounds__(256, BGPU_MIXED_FWD_MINB) k_mixed_fwd(const MixedArgs m) {
    extern __shared__ __align__(16) uint32_t sm[];
    const MixedClass& k = m.classes[mixed_class(m, 0, blockIdx.x)];
    const uint32_t local = blockIdx.x - k.begin[0];
    const uint32_t bx = local % k.tiles, rest = local / k.tiles;
    const uint32_t by = rest % kNumPrimes, bz = rest / kNumPrimes;
    switch (k.log_n2) {
        case 2: fwd_cols_body<0, 2, 256>(k.fwd, bx, by, bz, sm); break;
        case 3: fwd_cols_body<0, 3, 256>(k.fwd, bx, by, bz, sm); break;
        case 4: fwd_cols_body<0, 4, 256>(k.fwd, bx, by, bz, sm); break;
        case 5: fwd_cols_body<0, 5, 256>(k.fwd, bx, by, bz, sm); break;
        case 6: fwd_cols_body<0, 6, 256>(k.fwd, bx, by, bz, sm); break;
        case 7: fwd_cols_body<0, 7, 256>(k.fwd, bx, by, bz, sm); break;
        case 8: fwd_cols_body<0, 8, 256>(k.fwd, bx, by, bz, sm); break;
        default: fwd_cols_body<0, 9, 256>(k.fwd, bx, by, bz, sm); break;
    }
}

template <int L1, bool SQR>
__device__ __forceinline__ void mixed_mid_row(const MixedClass& k, uint32_t local, uint32_t* sm) {
    constexpr int T = mid_threads(L1);
    constexpr int RPC = kMixedMidThreads / T;  // rows per CTA
    const uint32_t sub = threadIdx.x / T;
    const uint32_t row = local * RPC + sub;
    mid_rows_body<0, L1, T, SQR, (RPC > 1)>(k.mid, row % k.rows, row / k.rows, sm + sub * k.mid_words);
}

template <bool SQR>
__device__ __forceinline__ void mixed_mid_len(const MixedClass& k, uint32_t local, uint32_t* sm) {
    switch (k.log_n1) {
        case 3: mixed_mid_row<3, SQR>(k, local, sm); break;
        case 4: mixed_mid_row<4, SQR>(k, local, sm); break;
        case 5: mixed_mid_row<5, SQR>(k, local, sm); break;
        case 6: mixed_mid_row<6, SQR>(k, local, sm); break;
        case 7: mixed_mid_row<7, SQR>(k, local, sm); break;
        case 8: mixed_mid_row<8, SQR>(k, local, sm); break;
        default: mixed_mid_row<9, SQR>(k, local, sm); break;
    }
}

static_assert(kSbThreads == kMixedMidThreads, "schoolbook CTAs ride in the mixed row pass");

__global__ void __launch_bounds__(kMixedMidThreads, BGPU_MIXED_MID_MINB)
    k_mixed_mid(const MixedArgs m) {
    extern __shared__ __align__(16) uint32_t sm[];
    if (blockIdx.x >= m.ntt_blocks[1]) {  // a schoolbook product: no wait on the column pass
        schoolbook_body(m.school[blockIdx.x - m.ntt_blocks[1]], *reinterpret_cast<SbSmem*>(sm));
        return;
    }
    const uint32_t b = blockIdx.x;
    const MixedClass& k = m.classes[mixed_class(m, 1, b)];
    const uint32_t local = b - k.begin[1];
    if (k.square)
        mixed_mid_len<true>(k, local, sm);
    else
        mixed_mid_len<false>(k, local, sm);
}

static_assert(kKaThreads == kNumPrimes * 128, "Karatsuba CTAs ride in the mixed inverse pass");

__global__ void __launch_bounds__(kNumPrimes * 128) k_mixed_inv(const MixedArgs m) {
    extern __shared__ __align__(16) uint32_t sm[];
    if (blockIdx.x >= m.ntt_blocks[2]) {  // a Karatsuba product: no wait on the row pass
        karatsuba_body(m.kara[blockIdx.x - m.ntt_blocks[2]], *reinterpret_cast<KaSmem*>(sm));
        return;
    }
    const uint32_t b = blockIdx.x;
    const MixedClass& k = m.classes[mixed_class(m, 2, b)];
    const uint32_t local = b - k.begin[2];
    const uint32_t bx = local % k.tiles, by = local / k.tiles;
    switch (k.log_n2) {
        case 2: inv_cols_body<0, 2, 128>(k.inv, bx, by, sm); break;
        case 3: inv_cols_body<0, 3, 128>(k.inv, bx, by, sm); break;
        case 4: inv_cols_body<0, 4, 128>(k.inv, bx, by, sm); break;
        case 5: inv_cols_body<0, 5, 128>(k.inv, bx, by, sm); break;
        case 6: inv_cols_body<0, 6, 128>(k.inv, bx, by, sm); break;
        case 7: inv_cols_body<0, 7, 128>(k.inv, bx, by, sm); break;
        case 8: inv_cols_body<0, 8, 128>(k.inv, bx, by, sm); break;
        default: inv_cols_body<0, 9, 128>(k.inv, bx, by, sm); break;
    }
}

__global__ void __launch_bounds__(kCarryThreads) k_mixed_carry(const MixedArgs m) {
    __shared__ uint32_t s_t;
    if (threadIdx.x == 0) s_t = (uint32_t)(atomicAdd(m.ticket, 1ull) - m.ticket_base);
    __syncthreads();
    pdl_wait();
    pdl_trigger();
    if (s_t >= gridDim.x) {  // the ticket counter and the launch disagree: report, touch nothing
        if (threadIdx.x == 0) atomicOr(m.err, 2u);
        return;
    }
    const MixedClass& k = m.classes[mixed_class(m, 3, s_t)];
    const uint32_t local = s_t - k.begin[3];
    carry_block<kCarryThreads, kCarryPer>(k.fwd.descs[local / k.bpp], local % k.bpp, k.nchunks, kFmtLimb64, m.epoch,
                                          m.err);
}

bool mixed_class_ok(int log_n, bool square) {
    const TransformShape sh = choose_shape_batch(log_n);
    return shape_ok(sh, square) && prime_set_for(log_n) == 0 && sh.log_n2 <= 9 && sh.log_n1 <= 9;
}

int mixed_fill(MixedClass* classes, int nclasses, const MixedClassSpec* spec, int slot, const NttConsts& c,
               MixedSizes* sizes) {
    if (nclasses > kMaxMixedClasses) return -1;
    uint32_t at[4] = {0, 0, 0, 0};
    size_t sm_fwd = 0, sm_mid = 0, sm_inv = 0;
    for (int i = 0; i < nclasses; ++i) {
        const MixedClassSpec& sp = spec[i];
        if (!mixed_class_ok(sp.log_n, sp.square)) return -1;
        const TransformShape sh = choose_shape_batch(sp.log_n);
        MixedClass& k = classes[i];
        k = MixedClass{};
        const int nops = sp.square ? 1 : 2;
        k.fwd.descs = sp.descs;
        k.fwd.nops = nops;
        k.fwd.log_n = sp.log_n;
        k.fwd.log_n1 = sh.log_n1;
        k.fwd.slot = slot;
        k.mid.descs = sp.descs;
        k.mid.log_n = sp.log_n;
        k.mid.log_n2 = sh.log_n2;
        k.mid.slot = slot;
        set_scale(c, sp.log_n, k.mid.scale_w, k.mid.scale_wp);
        k.inv.descs = sp.descs;
        k.inv.log_n = sp.log_n;
        k.inv.log_n1 = sh.log_n1;
        k.inv.slot = slot;
        k.tiles = (1u << sh.log_n1) / kCols;
        k.rows = 1u << sh.log_n2;
        k.count = sp.count;
        k.log_n1 = sh.log_n1;
        k.log_n2 = sh.log_n2;
        k.square = sp.square ? 1 : 0;
        k.nchunks = (uint32_t)(((size_t)1 << sp.log_n) / kCols);
        k.bpp = carry_blocks(k.nchunks);
        const uint32_t rpc = kMixedMidThreads / (uint32_t)mid_threads(sh.log_n1);
        const size_t row_bytes = (smem_mid_rows(sh.log_n1, sp.square) + 15) & ~(size_t)15;
        k.mid_words = (uint32_t)(row_bytes / 4);
        for (int pass = 0; pass < 4; ++pass) k.begin[pass] = at[pass];
        at[0] += k.tiles * kNumPrimes * nops * sp.count;
        at[1] += k.rows * kNumPrimes * sp.count / rpc;
        at[2] += k.tiles * sp.count;
        at[3] += k.bpp * sp.count;
        sm_fwd = std::max(sm_fwd, smem_fwd_cols(sh.log_n2, kCols));
        sm_mid = std::max(sm_mid, rpc * row_bytes);
        sm_inv = std::max(sm_inv, smem_inv_cols(sh.log_n2));
    }
    for (int pass = 0; pass < 4; ++pass) sizes->blocks[pass] = at[pass];
    sizes->smem[0] = sm_fwd;
    sizes->smem[1] = sm_mid;
    sizes->smem[2] = sm_inv;
    sizes->smem[3] = 0;
    return 0;
}

cudaError_t launch_ntt_mixed(const MixedArgs& m_in, const MixedSizes& sz, cudaStream_t st) {
    if (m_in.nclasses < 1) return cudaErrorInvalidValue;
    MixedArgs m = m_in;
    for (int pass = 0; pass < 4; ++pass) m.ntt_blocks[pass] = sz.blocks[pass];
    allow_smem(k_mixed_fwd, sz.smem[0]);
    cudaError_t e = launch_k(k_mixed_fwd, dim3(sz.blocks[0]), dim3(256), sz.smem[0], st, m);
    if (e != cudaSuccess) return e;
    const size_t sm_mid = std::max(sz.smem[1], m.nschool ? sizeof(SbSmem) : (size_t)0);
    allow_smem(k_mixed_mid, sm_mid);
    e = launch_k(k_mixed_mid, dim3(sz.blocks[1] + m.nschool), dim3(kMixedMidThreads), sm_mid, st, m);
    if (e != cudaSuccess) return e;
    const size_t sm_inv = std::max(sz.smem[2], m.nkara ? sizeof(KaSmem) : (size_t)0);
    allow_smem(k_mixed_inv, sm_inv);
    e = launch_k(k_mixed_inv, dim3(sz.blocks[2] + m.nkara), dim3(kNumPrimes * 128), sm_inv, st, m);
    if (e != cudaSuccess) return e;
    return launch_k(k_mixed_carry, dim3(sz.blocks[3]), dim3(kCarryThreads), 0, st, m);
}

const char* const kNttKernelNames[kNttLaunches] = {"k_fwd_cols", "k_mid_rows", "k_inv_cols",
                                                   "k_carry"};

}  // namespace bgpu
