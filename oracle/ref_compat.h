/* Force-included (g++ -include) when compiling the reference sources for the
 * CPU oracle library oracle/_ref/libbigint_ref.so.  The reference targets
 * MinGW, where size_t is `unsigned long long`; on Linux/x86-64 it is
 * `unsigned long`, so four call sites that mix `ull`/`ll` literals with
 * size_t/int64_t inside a single-template-parameter call fail deduction:
 *   include/bigint/mul.h:248            ceil_div((n - offset) * DIGIT_BITS, 64ull)
 *   src/bigint.cpp:94                   std::max(2ull, DEC_STRING_BRUTE_THRESHOLDS[0])
 *   src/bigint.cpp:983                  std::max(0ll, point_pos_)
 *   src/mul/ntt_multithread.cpp:40,91,121,150  std::max(1ull, total / ...)
 * Instead of editing (or copying) the reference, these non-template
 * overloads give each mixed call an exact match; values are unchanged
 * because both types are 64 bits wide here.  Test infrastructure only. */
#pragma once
#ifdef __cplusplus
#include <cstddef>
#include <cstdint>
#include <type_traits>
static_assert(sizeof(unsigned long) == sizeof(unsigned long long), "LP64 expected");
namespace std {
inline constexpr unsigned long long max(unsigned long long a, unsigned long b) {
    return a < b ? static_cast<unsigned long long>(b) : a;
}
inline constexpr long long max(long long a, long b) {
    return a < b ? static_cast<long long>(b) : a;
}
}  // namespace std
namespace bigint {
inline constexpr unsigned long ceil_div(unsigned long a, unsigned long long b) {
    return static_cast<unsigned long>(a / b + (a % b != 0));
}
}  // namespace bigint
#endif
