// Host-side construction of twiddle tables and constants (see tables.h).
#include "tables.h"

#include <cmath>

namespace bgpu {
namespace {

uint64_t pow_mod(uint64_t b, uint64_t e, uint64_t p) {
    uint64_t r = 1;
    b %= p;
    while (e) {
        if (e & 1) r = r * b % p;
        b = b * b % p;
        e >>= 1;
    }
    return r;
}

uint32_t inv32(uint32_t p) {  // p^-1 mod 2^32, p odd (Newton iteration)
    uint32_t x = 1;
    for (int i = 0; i < 5; ++i) x *= 2u - p * x;
    return x;
}

uint2 shoup_pair(uint64_t v, uint32_t p) {
    const uint32_t w = (uint32_t)(v % p);
    return make_uint2(w, (uint32_t)(((uint64_t)w << 32) / p));
}

uint2 mont_pair(uint64_t v, uint32_t p) {
    const uint32_t w = (uint32_t)(((v % p) << 32) % p);
    return make_uint2(w, w * inv32(p));
}

}  // namespace

void build_tables(int ps, int stage_log, uint2* host) {
    const PrimeSetInfo& s = kPrimeSets[ps];
    const size_t stage_n = (size_t)1 << stage_log;
    const size_t th_n = (size_t)1 << (s.log_max - s.split), tl_n = (size_t)1 << s.split;
    const size_t blk = table_block_entries(ps, stage_log);
    for (int q = 0; q < kNumPrimes; ++q) {
        const uint32_t p = s.p[q];
        for (int dir = 0; dir < 2; ++dir) {
            uint2* base = host + (size_t)(q * 2 + dir) * blk;
            base[0] = shoup_pair(1, p);
            for (size_t h = 1; h < stage_n; h <<= 1) {
                uint64_t root = pow_mod(s.g[q], (p - 1) / (2 * h), p);
                if (dir) root = pow_mod(root, p - 2, p);
                uint64_t v = 1;
                for (size_t m = 0; m < h; ++m) {
                    base[h + m] = shoup_pair(v, p);
                    v = v * root % p;
                }
            }
            uint64_t r = pow_mod(s.g[q], (p - 1) >> s.log_max, p);
            if (dir) r = pow_mod(r, p - 2, p);
            uint2* th = base + stage_n;
            uint2* tl = th + th_n;
            const uint64_t step_hi = pow_mod(r, tl_n, p);
            uint64_t v = 1;
            for (size_t i = 0; i < th_n; ++i, v = v * step_hi % p) th[i] = mont_pair(v, p);
            v = 1;
            for (size_t i = 0; i < tl_n; ++i, v = v * r % p) tl[i] = mont_pair(v, p);
        }
    }
}

// exp(sign * 2 pi i * num / den) rounded from long double.
static double2 root_of_unity(uint64_t num, uint64_t den, int sign) {
    const long double pi = 3.141592653589793238462643383279502884L;
    const long double ang = 2.0L * pi * (long double)num / (long double)den;
    return make_double2((double)cosl(ang), (double)(sign * sinl(ang)));
}

void build_fft_tables(double2* host) {
    const size_t stage_n = (size_t)1 << kFftStageLog;
    const size_t th_n = (size_t)1 << (kFftTwLog - kFftTwSplit), tl_n = (size_t)1 << kFftTwSplit;
    for (int dir = 0; dir < 2; ++dir) {
        const int sign = dir ? 1 : -1;  // forward uses exp(-2 pi i / N)
        double2* base = host + (size_t)dir * fft_table_block();
        base[0] = make_double2(1.0, 0.0);
        for (size_t h = 1; h < stage_n; h <<= 1)
            for (size_t m = 0; m < h; ++m) base[h + m] = root_of_unity(m, 2 * h, sign);
        double2* th = base + stage_n;
        double2* tl = th + th_n;
        const uint64_t full = (uint64_t)1 << kFftTwLog;
        for (size_t i = 0; i < th_n; ++i) th[i] = root_of_unity((uint64_t)i << kFftTwSplit, full, sign);
        for (size_t i = 0; i < tl_n; ++i) tl[i] = root_of_unity(i, full, sign);
    }
}

FftConsts make_fft_consts(const double2* dev_tables) {
    FftConsts c{};
    const size_t stage_n = (size_t)1 << kFftStageLog;
    const size_t th_n = (size_t)1 << (kFftTwLog - kFftTwSplit);
    for (int dir = 0; dir < 2; ++dir) {
        const double2* base = dev_tables + (size_t)dir * fft_table_block();
        c.stage[dir] = base;
        c.th[dir] = base + stage_n;
        c.tl[dir] = base + stage_n + th_n;
    }
    c.log_max = kFftTwLog;
    c.split = kFftTwSplit;
    return c;
}

NttConsts make_consts(int ps, int stage_log, const uint2* dev_tables) {
    const PrimeSetInfo& s = kPrimeSets[ps];
    NttConsts c{};
    const size_t stage_n = (size_t)1 << stage_log;
    const size_t th_n = (size_t)1 << (s.log_max - s.split);
    const size_t blk = table_block_entries(ps, stage_log);
    for (int q = 0; q < kNumPrimes; ++q) {
        const uint32_t p = s.p[q];
        c.pr[q].p = p;
        c.pr[q].pinv = inv32(p);
        const uint2 one = mont_pair(1, p);
        c.one_w[q] = one.x;
        c.one_wp[q] = one.y;
        c.red[q] = (uint32_t)(((uint64_t)1 << 32) / p);
        for (int dir = 0; dir < 2; ++dir) {
            const uint2* base = dev_tables + (size_t)(q * 2 + dir) * blk;
            c.stage[q][dir] = base;
            c.th[q][dir] = base + stage_n;
            c.tl[q][dir] = base + stage_n + th_n;
        }
    }
    const uint32_t p0 = s.p[0], p1 = s.p[1], p2 = s.p[2];
    const uint2 k1 = mont_pair(pow_mod(p0, p1 - 2, p1), p1);
    const uint2 k2 = mont_pair(p0 % p2, p2);
    const uint2 k3 = mont_pair(pow_mod((uint64_t)p0 * p1 % p2, p2 - 2, p2), p2);
    c.k1 = k1.x, c.k1p = k1.y;
    c.k2 = k2.x, c.k2p = k2.y;
    c.k3 = k3.x, c.k3p = k3.y;
    c.m01 = (uint64_t)p0 * p1;
    c.log_max = s.log_max;
    c.split = s.split;
    return c;
}

}  // namespace bgpu
