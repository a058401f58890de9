// Link-time hook that puts the reference's own BigInt / BigFloat code
// (Looading99/BigInt, unmodified) on top of this engine.
//
// The reference's multiply dispatch `_mul` is header-inline
// (include/bigint/mul.h:208-220) and calls three out-of-line functions: the
// NTT (src/mul/ntt_multithread.cpp:444), the FP64 FFT (src/mul/fft.cpp:281)
// and, above both, SSA (src/mul/ssa.cpp:383, whose leaves call _mul again).
// Building the reference WITHOUT ntt_multithread.cpp and fft.cpp and WITH
// this file makes every product that `_mul` does not keep on its inline
// schoolbook (total <= 16384 bits) run on the GPU through the C-ABI:
//   bigint::mul::ntt::mul  -> bgpu_mul_u64 (the engine's choice of method)
//   bigint::mul::fft::mul  -> bgpu_mul_u64 (exact for any size, unlike the
//                             reference's table-bounded FFT)
//   bigint::init_thread_pool -> bgpu_init (the engine replaces the CPU pool)
// Squaring is passed on by pointer identity, as the reference signals it.
// Errors surface as exceptions (std::bad_alloc for device memory, otherwise
// std::runtime_error): the reference's multiply cannot fail, so a failure
// here is never silent.
#include <cstdint>
#include <new>
#include <span>
#include <stdexcept>
#include <string>
#include <vector>

#include "bigint/bigint.h"
#include "bigint/mul.h"
#include "bigint_b200.h"

namespace {

void ensure_engine() {
    const int rc = bgpu_init(0);  // idempotent; device 0 unless the caller chose one
    if (rc != BGPU_OK) throw std::runtime_error(std::string("bigint_b200: ") + bgpu_strerror(rc));
}

std::vector<uint64_t> gpu_mul(std::span<const uint64_t> A, std::span<const uint64_t> B) {
    ensure_engine();
    std::vector<uint64_t> res(A.size() + B.size());
    size_t n = 0;
    // same data pointer and length: a square, as the reference detects it
    const int rc = bgpu_mul_u64(A.data(), A.size(), B.data(), B.size(), res.data(), res.size(), &n,
                                BGPU_METHOD_AUTO, nullptr);
    if (rc == BGPU_ERR_OOM) throw std::bad_alloc();
    if (rc != BGPU_OK) throw std::runtime_error(std::string("bigint_b200: ") + bgpu_strerror(rc));
    res.resize(n);  // no leading zero limbs, like the reference's ntt::mul / fft::mul
    return res;
}

}  // namespace

namespace bigint {

void init_thread_pool(uint32_t n) {
    (void)n;  // the GPU engine has no host thread pool
    ensure_engine();
}

namespace mul::ntt {
auto mul(std::span<const uint64_t> A, std::span<const uint64_t> B) -> std::vector<uint64_t> {
    return gpu_mul(A, B);
}
}  // namespace mul::ntt

namespace mul::fft {
auto mul(std::span<const uint64_t> A, std::span<const uint64_t> B, int digit_bits) -> std::vector<uint64_t> {
    (void)digit_bits;  // the engine picks the method; the product is exact either way
    return gpu_mul(A, B);
}
}  // namespace mul::fft

}  // namespace bigint
