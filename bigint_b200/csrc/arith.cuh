// Modular arithmetic for the three-prime NTT (device side).
//
// Primes (all < 2^31, 2^26 | p-1):
//   p0 = 469762049  = 7*2^26+1  (g = 3)   -- reference P[0] (ntt_base.h:15)
//   p1 = 1811939329 = 27*2^26+1 (g = 13)
//   p2 = 2013265921 = 15*2^27+1 (g = 31)  -- reference P[1]
// The reference's third prime 2281701377 > 2^31 is replaced by p1 so that every
// sum of two residues fits in 32 bits.  With 32-bit digits and N <= 2^26
// points every convolution coefficient is < min(da,db)*(2^32-1)^2 < 2^89
// < p0*p1*p2 (~2^90.47), so the CRT recovers each coefficient exactly and
// the integer product is identical to the reference's.
//
// Data is kept in normal (non-Montgomery) form, fully reduced to [0, p).
// Constants that multiply data are stored in Montgomery form w = c*2^32 mod p
// together with w' = w * p^-1 mod 2^32, so that
//   mont_mul_pre(a, w, w') = a * c  (mod p)   for any 32-bit a.
#pragma once
#include <cstdint>

namespace bgpu {

constexpr int kNumPrimes = 3;
constexpr int kMaxLogN = 26;   // largest transform: 2^26 points
constexpr int kMaxLogRow = 15; // stage twiddle table covers pair distances < 2^15
constexpr int kTwSplit = 13;   // inter-pass twiddle exponent split (2^26 = 2^13 * 2^13)

struct PrimeInfo {
    uint32_t p;
    uint32_t pinv;  // p^-1 mod 2^32
};

#ifdef __CUDACC__

__device__ __forceinline__ uint32_t mod_add(uint32_t a, uint32_t b, uint32_t p) {
    uint32_t s = a + b;  // < 2p < 2^32
    return min(s, s - p);
}

__device__ __forceinline__ uint32_t mod_sub(uint32_t a, uint32_t b, uint32_t p) {
    uint32_t d = a - b + p;  // in (0, 2p)
    return min(d, d - p);
}

// a * w * 2^-32 mod p with w' = w * p^-1 mod 2^32 precomputed; a < 2^32, w < p.
// hi(a*w) - hi(m*p) is exact because the low words of a*w and m*p agree.
__device__ __forceinline__ uint32_t mont_mul_pre(uint32_t a, uint32_t w, uint32_t wp, uint32_t p) {
    uint32_t m = a * wp;
    uint32_t h = __umulhi(a, w);
    uint32_t l = __umulhi(m, p);
    uint32_t r = h - l + p;  // in (0, 2p)
    return min(r, r - p);
}

// a * b * 2^-32 mod p, both operands variable (b < p).
__device__ __forceinline__ uint32_t mont_mul(uint32_t a, uint32_t b, uint32_t p, uint32_t pinv) {
    return mont_mul_pre(a, b, b * pinv, p);
}

#endif  // __CUDACC__

}  // namespace bgpu
