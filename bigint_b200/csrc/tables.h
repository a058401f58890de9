// Host-side twiddle tables and constants of one prime set.
//
// Per (prime q, direction d) the table block is
//   [stage: 2^stage_log Shoup pairs]  entry h+m = omega_{2h}^(+-m), h < 2^stage_log
//   [th: 2^(log_max-split) Montgomery pairs]  omega_{2^log_max}^(+-(i << split))
//   [tl: 2^split Montgomery pairs]            omega_{2^log_max}^(+-i)
// and the blocks are stored q-major, d-minor.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "engine.h"

namespace bgpu {

constexpr size_t table_block_entries(int ps, int stage_log) {
    return ((size_t)1 << stage_log) + ((size_t)1 << (kPrimeSets[ps].log_max - kPrimeSets[ps].split)) +
           ((size_t)1 << kPrimeSets[ps].split);
}

constexpr size_t table_entries(int ps, int stage_log) {
    return (size_t)kNumPrimes * 2 * table_block_entries(ps, stage_log);
}

// Fill `host` (table_entries(ps, stage_log) pairs).
void build_tables(int ps, int stage_log, uint2* host);

// FP64 twiddle tables of the FFT form: per direction [stage 2^kFftStageLog]
// [th 2^(kFftTwLog-kFftTwSplit)] [tl 2^kFftTwSplit] complex doubles.
constexpr size_t fft_table_block() {
    return ((size_t)1 << kFftStageLog) + ((size_t)1 << (kFftTwLog - kFftTwSplit)) +
           ((size_t)1 << kFftTwSplit);
}
void build_fft_tables(double2* host);  // 2 * fft_table_block() entries
FftConsts make_fft_consts(const double2* dev_tables);

// Constants of prime set `ps` whose table pointers point into `dev_tables`,
// a device copy of the host buffer built with the same (ps, stage_log).
NttConsts make_consts(int ps, int stage_log, const uint2* dev_tables);

}  // namespace bgpu
