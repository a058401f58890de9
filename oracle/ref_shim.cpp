// C-ABI shim over the UNMODIFIED reference multiply path (Looading99/BigInt),
// compiled together with the reference's own sources into
// oracle/_ref/libbigint_ref.so by oracle/build.py (build_ref).  It is test
// infrastructure: the parity tests, the golden-vector generator and the
// bench's CPU reference arm load it; the product never does.
//
// Every function forwards to one reference entry point:
//   ref_ntt_mul     -> bigint::mul::ntt::mul      src/mul/ntt_multithread.cpp:444
//   ref_fft_mul     -> bigint::mul::fft::mul      src/mul/fft.cpp:281
//   ref_ssa_mul     -> bigint::mul::ssa::mul      src/mul/ssa.cpp:383
//   ref_brute_mul   -> bigint::mul::brute::mul    include/bigint/mul.h:82
//   ref_mul         -> bigint::mul::_mul          include/bigint/mul.h:208
//   ref_mul_digits  -> bigint::mul::mul_digits    include/bigint/mul.h:223
//   ref_product_tree-> BigInt::operator* (bigint.h:284) over a pairwise tree
//   ref_fast_pow    -> bigint::fast_pow<BigInt>   include/bigint/bigint_base.h:60
//   ref_reciprocal  -> BigFloat::reciprocal       src/bigint.cpp:1044 (Newton, BigFloat::mul)
//   ref_bigfloat_reciprocal -> the same on BigFloat(x, offset), negated on request
//   ref_to_dec_string -> BigInt::print (decimal)  src/bigint.cpp:175-247
//   ref_from_dec_string -> BigInt(std::string)     src/bigint.cpp:25-124
//   ref_divmod      -> BigInt::divmod             src/bigint.cpp:625-673
//   ref_bigfloat_print -> BigFloat::print          src/bigint.cpp:972-1041
//   ref_init_thread_pool -> bigint::init_thread_pool (ntt_multithread.cpp:407)
// Results are copied into caller buffers; return 0 on success, -1 when the
// caller's buffer is too small (out_len then holds the needed size).
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <span>
#include <sstream>
#include <string>
#include <vector>

#include "bigint/bigint.h"
#include "bigint/mul.h"

namespace {

int copy_out64(const std::vector<uint64_t>& r, uint64_t* out, size_t cap, size_t* out_len) {
    *out_len = r.size();
    if (r.size() > cap) return -1;
    if (!r.empty()) std::memcpy(out, r.data(), r.size() * sizeof(uint64_t));
    return 0;
}

int copy_out32(const std::vector<uint32_t>& r, uint32_t* out, size_t cap, size_t* out_len) {
    *out_len = r.size();
    if (r.size() > cap) return -1;
    if (!r.empty()) std::memcpy(out, r.data(), r.size() * sizeof(uint32_t));
    return 0;
}

// The reference detects squaring by pointer identity (ntt_multithread.cpp:445,
// fft.cpp:283, mul.h:225); passing the same pointer for a and b reproduces it.
std::span<const uint64_t> span_b(const uint64_t* a, size_t na, const uint64_t* b, size_t nb) {
    if (a == b && na == nb) return std::span<const uint64_t>(a, na);
    return std::span<const uint64_t>(b, nb);
}

}  // namespace

extern "C" {

void ref_init_thread_pool(uint32_t n) { bigint::init_thread_pool(n); }

int ref_ntt_mul(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out,
                size_t cap, size_t* out_len) {
    auto r = bigint::mul::ntt::mul(std::span<const uint64_t>(a, na), span_b(a, na, b, nb));
    return copy_out64(r, out, cap, out_len);
}

int ref_fft_mul(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, int digit_bits,
                uint64_t* out, size_t cap, size_t* out_len) {
    auto r = bigint::mul::fft::mul(std::span<const uint64_t>(a, na), span_b(a, na, b, nb),
                                   digit_bits);
    return copy_out64(r, out, cap, out_len);
}

int ref_ssa_mul(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out,
                size_t cap, size_t* out_len) {
    auto r = bigint::mul::ssa::mul(std::span<const uint64_t>(a, na), span_b(a, na, b, nb));
    return copy_out64(r, out, cap, out_len);
}

int ref_brute_mul(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out,
                  size_t cap, size_t* out_len) {
    auto r = bigint::mul::brute::mul(std::span<const uint64_t>(a, na), span_b(a, na, b, nb));
    return copy_out64(r, out, cap, out_len);
}

int ref_mul(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out,
            size_t cap, size_t* out_len) {
    auto r = bigint::mul::_mul(std::span<const uint64_t>(a, na), span_b(a, na, b, nb));
    return copy_out64(r, out, cap, out_len);
}

// mul_digits takes `const Digits&`; squaring is `&a == &b`, so `same` != 0
// passes one vector twice.  point_pos may be null (the reference allows it).
int ref_mul_digits(const uint32_t* a, size_t na, const uint32_t* b, size_t nb, int same,
                   size_t output_precision, int64_t* point_pos, uint32_t* out, size_t cap,
                   size_t* out_len) {
    bigint::Digits da(a, a + na);
    if (same) {
        auto r = bigint::mul::mul_digits(da, da, output_precision, point_pos);
        return copy_out32(r, out, cap, out_len);
    }
    bigint::Digits db(b, b + nb);
    auto r = bigint::mul::mul_digits(da, db, output_precision, point_pos);
    return copy_out32(r, out, cap, out_len);
}

// Binary-splitting style product tree: leaves are u64 values; each level
// multiplies neighbours pairwise with BigInt::operator* (odd tail carried up).
// The product is returned as reference 28-bit Digits.
int ref_product_tree(const uint64_t* leaves, size_t n, uint32_t* out, size_t cap,
                     size_t* out_len) {
    std::vector<bigint::BigInt> level;
    level.reserve(n);
    for (size_t i = 0; i < n; ++i) level.emplace_back(leaves[i]);
    while (level.size() > 1) {
        std::vector<bigint::BigInt> next;
        next.reserve((level.size() + 1) / 2);
        for (size_t i = 0; i + 1 < level.size(); i += 2) next.push_back(level[i] * level[i + 1]);
        if (level.size() % 2) next.push_back(std::move(level.back()));
        level = std::move(next);
    }
    if (level.empty()) {
        *out_len = 0;
        return 0;
    }
    return copy_out32(level[0].get_data(), out, cap, out_len);
}

// 1 / x to `precision` digits for x = the product of `n` u64 leaves (built
// with BigInt::operator*, as ref_product_tree): the Newton iteration of
// BigFloat::reciprocal, whose products go through BigFloat::mul -> mul_digits.
// Returns the digits and the point position of the reciprocal.
int ref_reciprocal(const uint64_t* leaves, size_t n, size_t precision, uint32_t* out, size_t cap,
                   size_t* out_len, int64_t* point_pos) {
    bigint::BigInt x(1);
    for (size_t i = 0; i < n; ++i) x *= bigint::BigInt(leaves[i]);
    const bigint::BigFloat r = bigint::BigFloat(x).reciprocal(precision);
    *point_pos = r.get_point_pos();
    return copy_out32(r.get_data(), out, cap, out_len);
}

// BigFloat::reciprocal of +-BigFloat(X, offset) (the constructor of
// include/bigint/bigint.h:382: X * 2^offset, tail zeros removed), X given by
// its little-endian u64 limbs and built through the reference's hex-string
// constructor (src/bigint.cpp:25).  Returns the input BigFloat's digits,
// point position and sign as well, so a caller can hand the same BigFloat to
// another implementation.
int ref_bigfloat_reciprocal(const uint64_t* limbs, size_t n, int64_t offset, int neg, size_t precision,
                            uint32_t* in_out, size_t in_cap, size_t* in_len, int64_t* in_point_pos,
                            uint32_t* out, size_t cap, size_t* out_len, int64_t* point_pos, int* out_neg) {
    static const char hexd[] = "0123456789abcdef";
    std::string hex;
    hex.reserve(16 * n);
    for (size_t i = n; i-- > 0;)
        for (int k = 15; k >= 0; --k) hex.push_back(hexd[(limbs[i] >> (4 * k)) & 15]);
    bigint::BigInt x(hex, true);
    bigint::BigFloat v(x, offset);
    if (neg) v = -v;
    *in_point_pos = v.get_point_pos();
    if (copy_out32(v.get_data(), in_out, in_cap, in_len) != 0) return -1;
    const bigint::BigFloat r = v.reciprocal(precision);
    *point_pos = r.get_point_pos();
    *out_neg = r.sign() < 0 ? 1 : 0;
    return copy_out32(r.get_data(), out, cap, out_len);
}

// Decimal text of X (little-endian u64 limbs, built through the hex-string
// constructor, src/bigint.cpp:25) by BigInt::print (src/bigint.cpp:175-247,
// print_dec's divide-and-conquer over get_pow_of_ten and divmod).  Returns -1
// when cap is too small (out_len holds the size needed).
int ref_to_dec_string(const uint64_t* limbs, size_t n, char* out, size_t cap, size_t* out_len) {
    static const char hexd[] = "0123456789abcdef";
    std::string hex;
    hex.reserve(16 * n);
    for (size_t i = n; i-- > 0;)
        for (int k = 15; k >= 0; --k) hex.push_back(hexd[(limbs[i] >> (4 * k)) & 15]);
    bigint::BigInt x(hex, true);
    std::ostringstream os;
    x.print(os);
    const std::string s = os.str();
    *out_len = s.size();
    if (s.size() > cap) return -1;
    std::memcpy(out, s.data(), s.size());
    return 0;
}

// BigInt(const std::string&) (decimal; src/bigint.cpp:25-124): the Digits
// and the sign of the parsed number.
int ref_from_dec_string(const char* s, size_t len, uint32_t* out, size_t cap, size_t* out_len, int* neg) {
    const bigint::BigInt x(std::string(s, len), false);
    *neg = x.sign() < 0 ? 1 : 0;
    return copy_out32(x.get_data(), out, cap, out_len);
}

// a.divmod(b, mode, check) (src/bigint.cpp:625-673) for A and B given by
// little-endian u64 limbs (built through the hex-string constructor) and
// signs: the quotient's and the remainder's Digits and signs.  The caller
// keeps |A / B| away from [2^-28, 1], where the reference's conversion of the
// quotient estimate leaves an empty digit vector (undefined behaviour).
int ref_divmod(const uint64_t* a, size_t na, int a_neg, const uint64_t* b, size_t nb, int b_neg,
               uint32_t mode, int check, uint32_t* q, size_t q_cap, size_t* q_len, int* q_neg,
               uint32_t* r, size_t r_cap, size_t* r_len, int* r_neg) {
    static const char hexd[] = "0123456789abcdef";
    auto make = [](const uint64_t* limbs, size_t n, int neg) {
        std::string hex;
        hex.reserve(16 * n);
        for (size_t i = n; i-- > 0;)
            for (int k = 15; k >= 0; --k) hex.push_back(hexd[(limbs[i] >> (4 * k)) & 15]);
        bigint::BigInt x(hex, true);
        return neg ? -x : x;
    };
    const bigint::BigInt A = make(a, na, a_neg), B = make(b, nb, b_neg);
    const auto [Q, R] = A.divmod(B, static_cast<bigint::RoundMode>(mode), check != 0);
    *q_neg = Q.sign() < 0 ? 1 : 0;
    *r_neg = R.sign() < 0 ? 1 : 0;
    const int rq = copy_out32(Q.get_data(), q, q_cap, q_len);
    const int rr = copy_out32(R.get_data(), r, r_cap, r_len);
    return rq != 0 || rr != 0 ? -1 : 0;
}

// BigFloat::print(out, dec_digits) (src/bigint.cpp:972-1041) of
// +-BigFloat(X, offset) (X * 2^offset, tail zeros removed; X by its
// little-endian u64 limbs through the hex-string constructor).  Returns the
// input BigFloat's digits and point position as well, and the text.
int ref_bigfloat_print(const uint64_t* limbs, size_t n, int64_t offset, int neg, size_t dec_digits,
                       uint32_t* in_out, size_t in_cap, size_t* in_len, int64_t* in_point_pos, char* out,
                       size_t cap, size_t* out_len) {
    static const char hexd[] = "0123456789abcdef";
    std::string hex;
    hex.reserve(16 * n);
    for (size_t i = n; i-- > 0;)
        for (int k = 15; k >= 0; --k) hex.push_back(hexd[(limbs[i] >> (4 * k)) & 15]);
    bigint::BigFloat v(bigint::BigInt(hex, true), offset);
    if (neg) v = -v;
    *in_point_pos = v.get_point_pos();
    if (copy_out32(v.get_data(), in_out, in_cap, in_len) != 0) return -1;
    std::ostringstream os;
    v.print(os, dec_digits);
    const std::string s = os.str();
    *out_len = s.size();
    if (s.size() > cap) return -1;
    std::memcpy(out, s.data(), s.size());
    return 0;
}

// fast_pow over BigInt, as the reference's benchmark example calls it
// (examples/benchmark.cpp:22); the power is returned as 28-bit Digits.
int ref_fast_pow(uint64_t base, uint32_t exponent, uint32_t* out, size_t cap, size_t* out_len) {
    bigint::BigInt a(base);
    a = bigint::fast_pow(a, exponent);
    return copy_out32(a.get_data(), out, cap, out_len);
}

}  // extern "C"
