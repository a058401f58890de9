// Device bodies of the small-product kernels (schoolbook and Karatsuba, one
// CTA per product), shared by their own launches (small_kernels.cu) and by
// the mixed-length batch launches (ntt_kernels.cu), which run them in CTAs of
// the same size with their shared memory carved from the launch's dynamic
// buffer.
//
// Schoolbook computes what the reference's brute::mul computes
// (include/bigint/mul.h:82-102); the reference has no Karatsuba.  On the GPU
// a product is built from column sums: column k is the 192-bit sum of the
// 64x64-bit products a_i b_j with i + j = k, each owned by one thread, and a
// block-wide carry resolution (below) turns the columns into limbs without a
// serial pass.
//
// Karatsuba works on the polynomial coefficients: with h = ceil(max(na,nb)/2),
// a = a1 x^h + a0, b = b1 x^h + b0 (x = 2^64), the coefficient sums a0 + a1 and
// b0 + b1 keep their 65th bit instead of carrying, so
//     a b = z2 x^2h + (z1 - z0 - z2) x^h + z0,   z0 = a0 b0, z2 = a1 b1,
//     z1 = (a0 + a1)(b0 + b1)
// holds column by column and z1 - z0 - z2 = a0 b1 + a1 b0 is never negative.
// Three half-size products replace four (3h^2 instead of 4h^2 multiplies).
#pragma once
#include "engine.h"

namespace bgpu {

// (x2:x1:x0) += u * v
__device__ __forceinline__ void mac192(uint64_t& x0, uint64_t& x1, uint64_t& x2, uint64_t u, uint64_t v) {
    const uint64_t lo = u * v, hi = __umul64hi(u, v);
    x0 += lo;
    const uint64_t c = x0 < lo;
    const uint64_t t = x1 + hi;
    x2 += (t < x1);
    x1 = t + c;
    x2 += (x1 < c);
}

// (x2:x1) += v  (v added at the 2^64 position)
__device__ __forceinline__ void add_hi(uint64_t& x1, uint64_t& x2, uint64_t v) {
    x1 += v;
    x2 += (x1 < v);
}

// Low 64 bits and the (<= 2) overflow of c0[k] + c1[k-1] + c2[k-2]; zero
// outside [0, ncs).
__device__ __forceinline__ void column_word(const uint64_t* c0, const uint64_t* c1, const uint64_t* c2,
                                            int k, int ncs, uint64_t& lo, uint32_t& hi) {
    const uint64_t a = (k >= 0 && k < ncs) ? c0[k] : 0;
    const uint64_t b = (k >= 1 && k - 1 < ncs) ? c1[k - 1] : 0;
    const uint64_t c = (k >= 2 && k - 2 < ncs) ? c2[k - 2] : 0;
    uint64_t s = a + b;
    uint32_t h = s < a;
    const uint64_t t = s + c;
    h += t < s;
    lo = t;
    hi = h;
}

// Block-wide carry resolution: out[k], k < nout, are the limbs of
// sum_k (c2[k]:c1[k]:c0[k]) 2^(64k) over the ncs column sums.  Limb k is
//   L_k + H_{k-1} + carries,  (H_k:L_k) = c0[k] + c1[k-1] + c2[k-2],  H_k <= 2.
// v_k = L_k + H_{k-1} overflows by o_k <= 1; w_k = (v_k mod 2^64) + o_{k-1}
// overflows by g_k <= 1; what is left is a one-bit carry chain with generate
// g_k and propagate (w_k == 2^64 - 1), scanned with warp ballots and a fold
// over warps.  Every thread of the block must call it; s_wg/s_wp hold T/32
// words each.  P consecutive limbs per thread, T*P >= nout.
template <int T, int P>
__device__ __forceinline__ void block_resolve(const uint64_t* c0, const uint64_t* c1, const uint64_t* c2, int ncs,
                              int nout, uint64_t* out, uint32_t* s_wg, uint32_t* s_wp) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int k0 = threadIdx.x * P;
    uint64_t w[P];
    uint32_t g[P], pr[P];
    uint64_t lprev;
    uint32_t hprev, hprev2;
    {
        uint64_t l2;
        column_word(c0, c1, c2, k0 - 2, ncs, l2, hprev2);
        column_word(c0, c1, c2, k0 - 1, ncs, lprev, hprev);
    }
    // o_{k0-1}: overflow of L_{k0-1} + H_{k0-2}
    uint32_t oprev = (lprev + hprev2) < lprev;
#pragma unroll
    for (int i = 0; i < P; ++i) {
        uint64_t l;
        uint32_t h;
        column_word(c0, c1, c2, k0 + i, ncs, l, h);
        const uint64_t v = l + hprev;
        const uint32_t o = v < l;
        const uint64_t ww = v + oprev;
        g[i] = ww < v;
        pr[i] = (ww == ~0ull);
        w[i] = ww;
        if (k0 + i >= nout) {  // past the end: pass carries through
            g[i] = 0;
            pr[i] = 1;
        }
        hprev = h;
        oprev = o;
    }
    uint32_t G = 0, Pp = 1;
#pragma unroll
    for (int i = 0; i < P; ++i) {
        G = g[i] | (pr[i] & G);
        Pp &= pr[i];
    }
    const uint32_t gm = __ballot_sync(0xffffffffu, G);
    const uint32_t pm = __ballot_sync(0xffffffffu, Pp);
    const uint32_t bm = gm | pm;
    if (lane == 0) {
        s_wg[warp] = (uint32_t)((((uint64_t)gm + bm) >> 32) & 1u);
        s_wp[warp] = pm == 0xffffffffu;
    }
    __syncthreads();
    uint32_t cw = 0;
    for (int x = 0; x < warp; ++x) cw = s_wg[x] | (s_wp[x] & cw);
    const uint64_t sum = (uint64_t)gm + bm + cw;
    uint32_t c = (((uint32_t)sum ^ gm ^ bm) >> lane) & 1u;
#pragma unroll
    for (int i = 0; i < P; ++i) {
        if (k0 + i < nout) out[k0 + i] = w[i] + c;
        c = g[i] | (pr[i] & c);
    }
}

// ---- schoolbook --------------------------------------------------------------

constexpr int kSbThreads = 128;

// Shared memory of one schoolbook CTA.
struct SbSmem {
    uint64_t sa[kSchoolbookMaxLimbs], sb[kSchoolbookMaxLimbs];
    uint64_t c0[kSchoolbookMaxLimbs], c1[kSchoolbookMaxLimbs], c2[kSchoolbookMaxLimbs];
    uint32_t s_wg[kSbThreads / 32], s_wp[kSbThreads / 32];
};

// One product (na + nb <= kSchoolbookMaxLimbs) by one CTA of kSbThreads.
__device__ __forceinline__ void schoolbook_body(const SchoolDesc& d, SbSmem& S) {
    uint64_t* sa = S.sa;
    uint64_t* sb = S.sb;
    uint64_t* c0 = S.c0;
    uint64_t* c1 = S.c1;
    uint64_t* c2 = S.c2;
    uint32_t* s_wg = S.s_wg;
    uint32_t* s_wp = S.s_wp;
    for (uint32_t i = threadIdx.x; i < d.na; i += kSbThreads) sa[i] = d.a[i];
    for (uint32_t i = threadIdx.x; i < d.nb; i += kSbThreads) sb[i] = d.b[i];
    __syncthreads();
    const int ncs = (int)(d.na + d.nb) - 1;  // columns 0 .. na+nb-2
    for (int k = threadIdx.x; k < ncs; k += kSbThreads) {
        uint64_t x0 = 0, x1 = 0, x2 = 0;
        const int i0 = k + 1 > (int)d.nb ? k + 1 - (int)d.nb : 0;
        const int i1 = k < (int)d.na - 1 ? k : (int)d.na - 1;
        for (int i = i0; i <= i1; ++i) mac192(x0, x1, x2, sa[i], sb[k - i]);
        c0[k] = x0, c1[k] = x1, c2[k] = x2;
    }
    __syncthreads();
    block_resolve<kSbThreads, kSchoolbookMaxLimbs / kSbThreads>(c0, c1, c2, ncs, (int)(d.na + d.nb),
                                                                d.out, s_wg, s_wp);
}

// ---- Karatsuba ---------------------------------------------------------------

constexpr int kKaThreads = 384;           // 3 * (max h), one column pair per thread
constexpr int kKaHalf = kKaratsubaMaxLimbs / 2;  // largest h

// Shared memory of one Karatsuba CTA.
struct KaSmem {
    uint64_t A[2 * kKaHalf], B[2 * kKaHalf];  // operands, zero padded to 2h
    uint64_t SA[kKaHalf], SB[kKaHalf];        // a0 + a1, b0 + b1 (low words)
    uint64_t Z[3][3][2 * kKaHalf];            // [z0, z1, z2][word][column]
    uint64_t C[3][4 * kKaHalf];               // combined column sums
    uint8_t SAh[kKaHalf], SBh[kKaHalf];       // the sums' 65th bits
    uint32_t s_wg[kKaThreads / 32], s_wp[kKaThreads / 32];
};

// One product (na, nb <= kKaratsubaMaxLimbs) by one CTA of kKaThreads.
__device__ __forceinline__ void karatsuba_body(const SchoolDesc& d, KaSmem& S) {
    uint64_t* A = S.A;
    uint64_t* B = S.B;
    uint64_t* SA = S.SA;
    uint64_t* SB = S.SB;
    uint8_t* SAh = S.SAh;
    uint8_t* SBh = S.SBh;
    auto& Z = S.Z;
    auto& C = S.C;
    uint32_t* s_wg = S.s_wg;
    uint32_t* s_wp = S.s_wp;
    const int h = (int)((d.na > d.nb ? d.na : d.nb) + 1) / 2;
    for (int i = threadIdx.x; i < 2 * h; i += kKaThreads) {
        A[i] = i < (int)d.na ? d.a[i] : 0;
        B[i] = i < (int)d.nb ? d.b[i] : 0;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < h; i += kKaThreads) {
        const uint64_t x = A[i] + A[i + h], y = B[i] + B[i + h];
        SA[i] = x;
        SAh[i] = x < A[i];
        SB[i] = y;
        SBh[i] = y < B[i];
    }
    __syncthreads();
    // Column sums of the three h x h products: thread t takes product t / h
    // and the columns j and j + h (j = t mod h), h multiply-adds in all.
    if (threadIdx.x < 3 * h) {
        const int zp = threadIdx.x / h, j = threadIdx.x % h;
        for (int pass = 0; pass < 2; ++pass) {
            const int k = j + pass * h;
            if (k > 2 * h - 2) break;
            const int i0 = k - h + 1 > 0 ? k - h + 1 : 0;
            const int i1 = k < h - 1 ? k : h - 1;
            uint64_t x0 = 0, x1 = 0, x2 = 0;
            if (zp == 0) {
                for (int i = i0; i <= i1; ++i) mac192(x0, x1, x2, A[i], B[k - i]);
            } else if (zp == 2) {
                for (int i = i0; i <= i1; ++i) mac192(x0, x1, x2, A[h + i], B[h + k - i]);
            } else {
                // (x + X 2^64)(y + Y 2^64) = xy + (X y + Y x) 2^64 + X Y 2^128
                for (int i = i0; i <= i1; ++i) {
                    const uint64_t x = SA[i], y = SB[k - i];
                    const uint32_t X = SAh[i], Y = SBh[k - i];
                    mac192(x0, x1, x2, x, y);
                    if (X) add_hi(x1, x2, y);
                    if (Y) add_hi(x1, x2, x);
                    x2 += X & Y;
                }
            }
            Z[zp][0][k] = x0, Z[zp][1][k] = x1, Z[zp][2][k] = x2;
        }
    }
    __syncthreads();
    // Combine: C[K] = z0[K] + (z1 - z0 - z2)[K - h] + z2[K - 2h].
    const int nz = 2 * h - 1, ncs = 4 * h - 1;
    for (int K = threadIdx.x; K < ncs; K += kKaThreads) {
        uint64_t r0 = 0, r1 = 0, r2 = 0;
        if (K < nz) r0 = Z[0][0][K], r1 = Z[0][1][K], r2 = Z[0][2][K];
        if (K >= 2 * h) {
            const int m = K - 2 * h;
            const uint64_t t0 = r0 + Z[2][0][m];
            const uint64_t cy0 = t0 < r0;
            const uint64_t t1 = r1 + Z[2][1][m];
            const uint64_t cy1 = t1 < r1;
            const uint64_t t1c = t1 + cy0;
            r2 = r2 + Z[2][2][m] + cy1 + (t1c < t1);
            r0 = t0, r1 = t1c;
        }
        if (K >= h && K - h < nz) {
            const int m = K - h;
            // mid = z1 - z0 - z2 (non-negative column by column)
            uint64_t m0 = Z[1][0][m], m1 = Z[1][1][m], m2 = Z[1][2][m];
#pragma unroll
            for (int s = 0; s < 3; s += 2) {
                const uint64_t b0 = Z[s][0][m], b1 = Z[s][1][m], b2 = Z[s][2][m];
                const uint64_t u0 = m0 - b0;
                const uint64_t br0 = m0 < b0;
                const uint64_t u1 = m1 - b1;
                const uint64_t br1 = m1 < b1;
                const uint64_t u1b = u1 - br0;
                const uint64_t br1b = u1 < br0;
                m2 = m2 - b2 - br1 - br1b;
                m0 = u0, m1 = u1b;
            }
            const uint64_t t0 = r0 + m0;
            const uint64_t cy0 = t0 < r0;
            const uint64_t t1 = r1 + m1;
            const uint64_t cy1 = t1 < r1;
            const uint64_t t1c = t1 + cy0;
            r2 = r2 + m2 + cy1 + (t1c < t1);
            r0 = t0, r1 = t1c;
        }
        C[0][K] = r0, C[1][K] = r1, C[2][K] = r2;
    }
    __syncthreads();
    block_resolve<kKaThreads, (2 * kKaratsubaMaxLimbs + kKaThreads - 1) / kKaThreads>(
        C[0], C[1], C[2], ncs, (int)(d.na + d.nb), d.out, s_wg, s_wp);
}

}  // namespace bgpu
