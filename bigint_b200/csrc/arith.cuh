// Modular arithmetic for the three-prime NTT (device side) and the two prime
// sets the engine uses.
//
// Set 0 ("lazy", transforms up to 2^23 points), all primes < 2^30:
//   469762049 = 7*2^26+1 (g 3), 754974721 = 45*2^24+1 (g 11), 998244353 = 119*2^23+1 (g 3)
//   product ~2^88.19.  With 32-bit digits and N <= 2^23 every coefficient is
//   < (N/2)(2^32-1)^2 < 2^86, so CRT is exact.  Because 4p < 2^32, residues
//   may stay unreduced in [0, 2p) / [0, 4p) between butterflies (Harvey's
//   lazy butterflies with Shoup multiplication): 7 instructions per butterfly.
// Set 1 ("strict", up to 2^26 points), all primes < 2^31:
//   469762049 (g 3), 1811939329 = 27*2^26+1 (g 13), 2013265921 = 15*2^27+1 (g 31)
//   product ~2^90.47 > 2^89 >= (N/2)(2^32-1)^2 for N <= 2^26; residues are
//   kept fully reduced in [0, p) (sums of two still fit in 32 bits).
// 469762049 and 2013265921 are the reference's own P[0], P[1]
// (include/bigint/ntt_base.h:15); its third prime 2281701377 > 2^31 would not
// leave room for carry-free sums.
//
// Twiddles of the butterflies are Shoup pairs (W, W' = floor(W 2^32 / p)),
// W in normal form.  Constants multiplying data elsewhere are Montgomery
// pairs (w = c 2^32 mod p, w' = w p^-1 mod 2^32): a*c = hi(a w) - hi((a w') p).
#pragma once
#include <cstdint>

namespace bgpu {

constexpr int kNumPrimes = 3;
constexpr int kNumSets = 2;
constexpr int kMaxLogN = 26;    // largest transform overall (set 1)
constexpr int kLazyMaxLogN = 23;  // largest transform of set 0
constexpr int kMaxLogRow = 15;  // stage tables cover pair distances h < 2^15

struct PrimeSetInfo {
    uint32_t p[kNumPrimes];
    uint32_t g[kNumPrimes];
    int log_max;  // 2^log_max | p-1 for every prime of the set
    int split;    // inter-pass twiddle exponent split: e = hi << split | lo
};

constexpr PrimeSetInfo kPrimeSets[kNumSets] = {
    {{469762049u, 754974721u, 998244353u}, {3u, 11u, 3u}, kLazyMaxLogN, 12},
    {{469762049u, 1811939329u, 2013265921u}, {3u, 13u, 31u}, kMaxLogN, 13},
};

inline int prime_set_for(int log_n) { return log_n <= kLazyMaxLogN ? 0 : 1; }

struct PrimeInfo {
    uint32_t p;
    uint32_t pinv;  // p^-1 mod 2^32
};

#ifdef __CUDACC__

__device__ __forceinline__ uint32_t umin(uint32_t a, uint32_t b) { return min(a, b); }

// x - m if x >= m else x, for x < 2m (and m <= 2^31): one add and one min.
__device__ __forceinline__ uint32_t csub(uint32_t x, uint32_t m) { return min(x, x - m); }

__device__ __forceinline__ uint32_t mod_add(uint32_t a, uint32_t b, uint32_t p) {
    return csub(a + b, p);  // a, b < p < 2^31
}

__device__ __forceinline__ uint32_t mod_sub(uint32_t a, uint32_t b, uint32_t p) {
    return csub(a - b + p, p);
}

// Shoup: x*W mod p lazily in [0, 2p) for any 32-bit x (W < p, W' = floor(W 2^32/p)).
__device__ __forceinline__ uint32_t shoup_lazy(uint32_t x, uint32_t w, uint32_t wp, uint32_t p) {
    const uint32_t q = __umulhi(x, wp);
    return x * w - q * p;
}

// Montgomery: a*w*2^-32 mod p lazily in (0, 2p) (a < 2^32, w < p, w' = w p^-1).
__device__ __forceinline__ uint32_t mont_lazy(uint32_t a, uint32_t w, uint32_t wp, uint32_t p) {
    const uint32_t m = a * wp;
    return __umulhi(a, w) - __umulhi(m, p) + p;
}

__device__ __forceinline__ uint32_t mont_mul_pre(uint32_t a, uint32_t w, uint32_t wp, uint32_t p) {
    return csub(mont_lazy(a, w, wp, p), p);
}

__device__ __forceinline__ uint32_t mont_mul(uint32_t a, uint32_t b, uint32_t p, uint32_t pinv) {
    return mont_mul_pre(a, b, b * pinv, p);
}

// Butterflies.  LAZY: DIF takes/returns [0, 2p); DIT takes [0, 4p) and
// returns [0, 4p).  Strict: everything in [0, p).
template <bool LAZY>
struct Bfly;

template <>
struct Bfly<true> {
    // (a, b) -> (a + b, (a - b) W)
    static __device__ __forceinline__ void dif(uint32_t& a, uint32_t& b, uint32_t w, uint32_t wp,
                                               uint32_t p) {
        const uint32_t p2 = 2 * p;
        const uint32_t s = csub(a + b, p2);
        const uint32_t t = a - b + p2;
        b = shoup_lazy(t, w, wp, p);
        a = s;
    }
    static __device__ __forceinline__ void dif1(uint32_t& a, uint32_t& b, uint32_t p) {
        const uint32_t p2 = 2 * p;
        const uint32_t s = csub(a + b, p2);
        b = csub(a - b + p2, p2);
        a = s;
    }
    // (a, b) -> (a + b W, a - b W)
    static __device__ __forceinline__ void dit(uint32_t& a, uint32_t& b, uint32_t w, uint32_t wp,
                                               uint32_t p) {
        const uint32_t p2 = 2 * p;
        const uint32_t x = csub(a, p2);
        const uint32_t t = shoup_lazy(b, w, wp, p);
        a = x + t;
        b = x - t + p2;
    }
    static __device__ __forceinline__ void dit1(uint32_t& a, uint32_t& b, uint32_t p) {
        const uint32_t p2 = 2 * p;
        const uint32_t x = csub(a, p2);
        const uint32_t t = csub(b, p2);
        a = x + t;
        b = x - t + p2;
    }
    // reduce a butterfly output to [0, p)
    static __device__ __forceinline__ uint32_t reduce(uint32_t x, uint32_t p) {
        return csub(csub(x, 2 * p), p);
    }
};

template <>
struct Bfly<false> {
    static __device__ __forceinline__ void dif(uint32_t& a, uint32_t& b, uint32_t w, uint32_t wp,
                                               uint32_t p) {
        const uint32_t s = mod_add(a, b, p);
        const uint32_t t = a - b + p;  // (0, 2p), any 32-bit input is fine for Shoup
        b = csub(shoup_lazy(t, w, wp, p), p);
        a = s;
    }
    static __device__ __forceinline__ void dif1(uint32_t& a, uint32_t& b, uint32_t p) {
        const uint32_t s = mod_add(a, b, p);
        b = mod_sub(a, b, p);
        a = s;
    }
    static __device__ __forceinline__ void dit(uint32_t& a, uint32_t& b, uint32_t w, uint32_t wp,
                                               uint32_t p) {
        const uint32_t t = csub(shoup_lazy(b, w, wp, p), p);
        b = mod_sub(a, t, p);
        a = mod_add(a, t, p);
    }
    static __device__ __forceinline__ void dit1(uint32_t& a, uint32_t& b, uint32_t p) {
        const uint32_t t = b;
        b = mod_sub(a, t, p);
        a = mod_add(a, t, p);
    }
    static __device__ __forceinline__ uint32_t reduce(uint32_t x, uint32_t) { return x; }
};

#endif  // __CUDACC__

}  // namespace bgpu
