/* bigint_b200 -- C-ABI of the B200 big-integer multiply engine.
 *
 * Drop-in boundary for the multiply path of Looading99/BigInt.  Each entry
 * point states the reference interface it replaces (paths inside that
 * project).  All functions are plain C: host pointers and sizes in, status
 * code out; they never throw.  Device-pointer variants take a CUDA stream as
 * `void*`.  Unless noted, calls are serialized by an internal mutex, like the
 * reference's pool (src/mul/ntt_multithread.cpp:259-260).
 *
 * Conventions shared with the reference:
 *  - u64 limbs and 28-bit Digits are little-endian.
 *  - squaring is signalled by passing the SAME pointer (and length) for both
 *    operands, as the reference detects it by address
 *    (include/bigint/mul.h:225, src/mul/ntt_multithread.cpp:445).
 *  - results carry no leading zero limbs/digits.
 */
#ifndef BIGINT_B200_H
#define BIGINT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes (0 = success). */
#define BGPU_OK 0
#define BGPU_ERR_INVALID_ARG -1   /* null pointer, zero length, digit >= 2^28 ... */
#define BGPU_ERR_NO_DEVICE -2     /* no CUDA device / CUDA runtime error at init */
#define BGPU_ERR_OOM -3           /* device or pinned-host allocation failed */
#define BGPU_ERR_CAPACITY -4      /* size beyond what the entry point supports */
#define BGPU_ERR_OUT_CAPACITY -5  /* caller's output buffer too small; *out_len = needed */
#define BGPU_ERR_CUDA -6          /* CUDA error during the multiply */
#define BGPU_ERR_DEVICE_TIMEOUT -7/* a bounded device-side wait gave up (carry look-back), or the
                                     carry scan saw a block ticket outside its launch */
#define BGPU_ERR_NOT_INIT -8      /* bgpu_init() not called / failed */

/* Method selection (flags & BGPU_METHOD_MASK). */
#define BGPU_METHOD_AUTO 0u
#define BGPU_METHOD_NTT 1u        /* three-prime NTT (the plain method) */
#define BGPU_METHOD_SCHOOLBOOK 2u /* O(n*m) kernel; na + nb <= BGPU_SCHOOLBOOK_MAX_LIMBS */
#define BGPU_METHOD_FFT 3u        /* FP64 complex FFT (bgpu_mul_u64 only); products whose
                                     max |x - round(x)| exceeds 1/4 are redone on the NTT */
#define BGPU_METHOD_KARATSUBA 4u  /* one Karatsuba level over column sums; na, nb each
                                     <= BGPU_KARATSUBA_MAX_LIMBS (no counterpart in the
                                     reference, whose brute::mul is plain schoolbook) */
#define BGPU_METHOD_MASK 0xFu
/* FFT form: choose bits per point from the average-case error growth instead
 * of the worst-case bound (more bits, runtime check + NTT fallback). */
#define BGPU_FFT_AVERAGE_BOUND 0x10u
/* FFT form: force b bits per point (8..20) in flags bits 8..12. */
#define BGPU_FFT_BITS(b) ((uint32_t)(b) << 8)
/* bgpu_mul_u64_device only: the caller promises that nothing still running
 * or queued on the stream writes this product's operands (a stream of
 * independent products).  The transform of this product may then start while
 * the previous product's carry scan finishes; every later kernel still runs
 * after both.  Ignored when the operands overlap the previous call's output. */
#define BGPU_INDEPENDENT 0x20u
/* bgpu_batch_plan_create / bgpu_mul_batch_device: give every NTT class of the
 * batch its own four launches on parallel graph branches instead of one launch
 * per pass for all classes (see the batch plan section). */
#define BGPU_BATCH_PER_CLASS 0x40u

#define BGPU_SCHOOLBOOK_MAX_LIMBS 256u
#define BGPU_KARATSUBA_MAX_LIMBS 256u
#define BGPU_MAX_LOG2_POINTS 26u  /* transform points are 32-bit digits */
/* Largest |point_pos| the BigFloat entry points take (BGPU_ERR_CAPACITY
 * above): 28 * point_pos then stays far inside int64_t. */
#define BGPU_MAX_POINT_POS ((int64_t)1 << 40)

typedef struct bgpu_stats {
    int32_t method;          /* BGPU_METHOD_* actually used */
    uint32_t log2_points;    /* transform length (0 for schoolbook) */
    double max_round_err;    /* FFT form: max |x - round(x)| over all coefficients; 0 otherwise */
    int32_t fell_back;       /* FFT form: 1 if the product was recomputed on the NTT */
    float device_ms;         /* device time of the multiply kernels */
    int32_t fft_bits;        /* FFT form: bits per point used */
} bgpu_stats;

/* Select the CUDA device and build the twiddle tables.  Idempotent; a second
 * call with another device re-initializes.  Replaces the reference's
 * init_thread_pool (include/bigint/bigint.h:35-38) as the engine set-up. */
int bgpu_init(int device);

/* Release device tables, scratch and streams. */
int bgpu_shutdown(void);

/* Human-readable text for a status code. */
const char* bgpu_strerror(int code);

/* Product of u64-limb integers: the `_mul` seam (include/bigint/mul.h:208-220)
 * and ntt::mul (src/mul/ntt_multithread.cpp:444-530).  Writes the product
 * without leading zeros into out[0..*out_len).  A zero operand gives
 * *out_len == 0 (brute::mul's result, include/bigint/mul.h:82-102).  Products
 * above 2^31 bits, beyond the largest transform (where the reference uses
 * ssa::mul, src/mul/ssa.cpp:383), run as blocks of 2^30-bit NTT products
 * added on the device; na + nb is limited to 2^31 limbs. */
int bgpu_mul_u64(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out,
                 size_t out_cap, size_t* out_len, uint32_t flags, bgpu_stats* stats);

/* Product of 28-bit Digits: the mul_digits seam (include/bigint/mul.h:223-318),
 * called from BigInt::operator* (include/bigint/bigint.h:289) and
 * BigFloat::mul (include/bigint/bigint.h:576).  Same output_precision /
 * point_pos semantics as the reference: with output_precision > 0 only the
 * top digits of each operand are used, the result is cut to about that many
 * digits and *point_pos is decreased by the digits dropped; with 0 the exact
 * product is returned (low zero digits re-inserted).  point_pos may be NULL.
 * Precondition as in the reference: neither operand is all zero
 * (BGPU_ERR_INVALID_ARG instead of undefined behaviour). */
int bgpu_mul_digits(const uint32_t* a, size_t na, const uint32_t* b, size_t nb,
                    size_t output_precision, int64_t* point_pos, uint32_t* out, size_t out_cap,
                    size_t* out_len, uint32_t flags, bgpu_stats* stats);

/* Many independent products of host-resident operands, pipelined: each
 * product's operands are copied to the GPU, multiplied and the product copied
 * back, with the copies of neighbouring products overlapping the multiply
 * (four device slots, separate copy streams).  The reference multiplies one
 * pair per call (_mul, include/bigint/mul.h:208-220); this is that call over a
 * list, for callers with many products at hand (binary splitting,
 * examples/pi.cpp:41-80).  out receives na + nb limbs (out_cap >= na + nb;
 * zero padded) and *out_len the length without leading zeros.  a == b with
 * na == nb squares.  Overlap needs page-locked host buffers; pageable ones
 * work but copy synchronously.  Returns after every product is back. */
typedef struct bgpu_host_product {
    const uint64_t* a;
    size_t na;
    const uint64_t* b;
    size_t nb;
    uint64_t* out;
    size_t out_cap;
    size_t* out_len;
} bgpu_host_product;
int bgpu_mul_u64_many(const bgpu_host_product* products, size_t count, uint32_t flags);

/* base^exponent for a u64-limb base: the reference's fast_pow<BigInt>
 * (include/bigint/bigint_base.h:60-69, the squaring chain its benchmark
 * example times, examples/benchmark.cpp:22), every product on the GPU with no
 * host round trip between them.  Writes the power without leading zeros;
 * 0^0 = 1 like the reference's res = 1.  Products beyond the largest
 * transform run as its blocks, as in bgpu_mul_u64; BGPU_ERR_CAPACITY when
 * the power exceeds 2^30 limbs. */
int bgpu_pow_u64(const uint64_t* base, size_t nbase, uint32_t exponent, uint64_t* out,
                 size_t out_cap, size_t* out_len);

/* BigInt to decimal text: the reference's BigInt::print (src/bigint.cpp:175-247,
 * print_dec).  The input is the BigInt's Digits (28-bit) and sign; writes the
 * text ('-' for a negative nonzero value, no leading zeros, "0" for zero),
 * identical to the reference's, not NUL-terminated.  The conversion runs on
 * the GPU: halves by 10^(19 * 2^k) top down, with exact reciprocals and
 * batched products, and leaves of 608 digits.  BGPU_ERR_OUT_CAPACITY when
 * out_cap is too small (*out_len = needed). */
int bgpu_to_decimal(const uint32_t* digits, size_t n, int is_neg, char* out, size_t out_cap, size_t* out_len);

/* Decimal text to a BigInt: the reference's BigInt(const std::string&) with
 * hex = false (src/bigint.cpp:25-90) and its convert_from_dec_string
 * (:92-124).  Characters before the first digit may hold '-' (the number is
 * then negative); characters that are not digits are skipped.  Writes the
 * BigInt's Digits (28-bit, no leading zeros; zero is the single digit 0, not
 * negative) and its sign.  The value is built on the GPU: 19-digit leaves
 * paired level by level through hi * 10^(19 * 2^j) + lo, every level one batch
 * of equal-size products.  Up to 19 * 2^25 digits (BGPU_ERR_CAPACITY above). */
int bgpu_from_decimal(const char* s, size_t len, uint32_t* out, size_t out_cap, size_t* out_len,
                      int* is_neg);

/* Reciprocal of a BigFloat: BigFloat::reciprocal(precision)
 * (src/bigint.cpp:1044-1071), its Newton iteration
 * x += mul(x, 1 - mul(b, x, p + 1), p + 1) run with every value on the GPU
 * (the truncated products of BigFloat::mul / mul_digits, the additions and
 * subtractions of BigFloat::add_or_sub, the shifts), so no digit array makes a
 * host round trip between steps.  The input is the BigFloat's fields: its
 * Digits (28-bit, no leading zero digit), point position (value = digits *
 * 2^(-28 point_pos)) and sign; precision 0 means the input's digit count, as
 * in the reference.  Writes the reciprocal's Digits, point position and sign,
 * identical to the reference's result.  Division by zero (the reference
 * throws std::domain_error) and digits >= 2^28 give BGPU_ERR_INVALID_ARG;
 * |point_pos| > BGPU_MAX_POINT_POS gives BGPU_ERR_CAPACITY;
 * BGPU_ERR_OUT_CAPACITY when out_cap is too small (*out_len = needed). */
int bgpu_reciprocal_digits(const uint32_t* digits, size_t n, int64_t point_pos, int is_neg,
                           size_t precision, uint32_t* out, size_t out_cap, size_t* out_len,
                           int64_t* out_point_pos, int* out_is_neg);

/* Decimal text of a BigFloat: the reference's BigFloat::print(out, dec_digits)
 * (src/bigint.cpp:972-1041) on the BigFloat's fields (Digits, point position,
 * sign).  The integer part prints as it is; the fraction f becomes
 * round_half_up(f * 10^d), with d = dec_digits (0: floor(28 * (fraction
 * digits) * log10 2), as in the reference), carried into the integer part when
 * it reaches 10^d, and prints padded to d digits: "[-]int.frac" (just "int."
 * when d is 0), identical to the reference's text, not NUL-terminated.  5^d,
 * the product, the shift, the rounding and both decimal conversions run on
 * the GPU.  Where the reference's rounding is undefined (2^-28 <= f * 10^d <
 * 1/2) the fraction prints as zeros.  |point_pos| > BGPU_MAX_POINT_POS gives
 * BGPU_ERR_CAPACITY; BGPU_ERR_OUT_CAPACITY when out_cap is too small
 * (*out_len = needed). */
int bgpu_bigfloat_to_decimal(const uint32_t* digits, size_t n, int64_t point_pos, int is_neg,
                             size_t dec_digits, char* out, size_t out_cap, size_t* out_len);

/* Quotient and remainder: the reference's BigInt::divmod(b, mode, check)
 * (src/bigint.cpp:625-673) on +-A and +-B given as Digits (28-bit, no leading
 * zeros; zero is the single digit 0) and signs.  The reference's steps run on
 * the GPU: the estimate BigFloat::mul(A, B.reciprocal(n_a + 16), n_a + 16)
 * rounded by `mode` (0 Truncate, 1 Floor, 2 Ceil, 3 RoundHalfUp; other values
 * below 256 act as Truncate, as in the reference), R = A - Q * B, and with
 * `check` one adjustment by +-1 when R breaks the mode's bound.  Writes Q's
 * and R's Digits and signs, identical to the reference's.  Where the
 * reference's conversion of the estimate is undefined (2^-28 <= |estimate| <
 * 1 with nothing added by the rounding), Q starts from zero.  B = 0 (the
 * reference throws std::domain_error), digits >= 2^28, a leading zero digit or
 * mode >= 256 give BGPU_ERR_INVALID_ARG; BGPU_ERR_OUT_CAPACITY when a buffer
 * is too small (*q_len and *r_len = the lengths needed). */
int bgpu_divmod_digits(const uint32_t* a, size_t na, int a_neg, const uint32_t* b, size_t nb, int b_neg,
                       uint32_t mode, int check, uint32_t* q, size_t q_cap, size_t* q_len, int* q_neg,
                       uint32_t* r, size_t r_cap, size_t* r_len, int* r_neg);

/* Device-resident product (no host copies, asynchronous on `stream`, a
 * cudaStream_t; 0 is the legacy default stream): d_out receives exactly
 * na + nb limbs (zero padded).  d_a == d_b with na == nb squares.  Errors
 * found on the device are sticky and reported by bgpu_device_status.  The
 * engine's scratch is shared: calls that overlap on the GPU (different
 * streams, or this and the host-buffer entry points at once) race. */
int bgpu_mul_u64_device(const uint64_t* d_a, size_t na, const uint64_t* d_b, size_t nb,
                        uint64_t* d_out, uint32_t flags, void* stream);

/* Synchronize `stream` (0 = legacy default stream) and return (and clear)
 * the sticky device status. */
int bgpu_device_status(void* stream);

/* Diagnostic of failure detection, safe to run on a shared GPU: one thread
 * runs the carry scan's bounded wait on a device flag word for at most
 * spin_limit polls.  With set_flag = 0 nothing ever sets the flag, the wait
 * gives up, the device error word is set and the call returns
 * BGPU_ERR_DEVICE_TIMEOUT (the context stays usable and the error is cleared);
 * with set_flag = 1 the flag is already set and the call returns BGPU_OK.
 * No counterpart in the reference (its waits are on host threads,
 * src/mul/ntt_multithread.cpp:184-203). */
int bgpu_selftest_wait(uint32_t spin_limit, int set_flag);

/* Number of kernel launches the last multiply issued (for bench accounting). */
uint32_t bgpu_last_launch_count(void);

/* Per-kernel device timing (CUDA events recorded between the launches of each
 * NTT product, on the stream the kernels run on).  No reference counterpart:
 * the reference has no tracing beyond std::chrono in its examples
 * (examples/benchmark.cpp:17-38). */
int bgpu_set_kernel_timing(int on);

/* Mean device time of each kernel over the NTT products launched since
 * timing was switched on (the last 1024 of them): names[i], mean_ms[i] in
 * launch order, *nproducts = products averaged.  Returns the kernel count
 * (0 if none recorded).  Synchronizes on the last recorded event. */
int bgpu_kernel_times(const char** names, float* mean_ms, int cap, uint32_t* nproducts);

/* ---- batches of independent products ----
 * The reference multiplies one pair per call; its binary-splitting caller
 * (examples/pi.cpp:41-80) and fast_pow produce many independent products per
 * step.  A plan groups a batch by size (schoolbook below
 * BGPU_SCHOOLBOOK_MAX_LIMBS, Karatsuba, then one NTT class per transform
 * length), allocates its scratch once and captures every launch of the batch
 * into one CUDA graph; running the plan is one graph launch.  A batch of
 * several transform lengths runs as one launch per NTT pass (four kernel
 * nodes holding every class's blocks, the small products riding in two of
 * them); with BGPU_BATCH_PER_CLASS every class gets its own four launches on
 * parallel graph branches, which overlap one another's pass boundaries (on a
 * B200 the 4096-product log-uniform batch ran 4.5 % faster that way, with 38
 * nodes instead of 4).  Pointers are device pointers; out receives na + nb
 * limbs; a == b with na == nb squares.  A plan is bound to the pointers it
 * was made with (rebuild it for new buffers). */
typedef struct bgpu_product {
    const uint64_t* a;
    size_t na;
    const uint64_t* b;
    size_t nb;
    uint64_t* out;
} bgpu_product;

typedef struct bgpu_batch_plan_s* bgpu_batch_plan;

int bgpu_batch_plan_create(const bgpu_product* products, size_t count, uint32_t flags,
                           bgpu_batch_plan* plan);
/* Launch the plan's graph on `stream` (asynchronous); device-side errors are
 * reported by bgpu_device_status.  Runs of one plan must not overlap. */
int bgpu_batch_plan_run(bgpu_batch_plan plan, void* stream);
int bgpu_batch_plan_destroy(bgpu_batch_plan plan);
/* Kernel launches one run of the plan makes (its graph's kernel nodes). */
uint32_t bgpu_batch_plan_launches(bgpu_batch_plan plan);
/* One-shot: create, run, synchronize, destroy. */
int bgpu_mul_batch_device(const bgpu_product* products, size_t count, uint32_t flags, void* stream);

/* Pairwise product tree of n u64 values (the binary-splitting pattern of
 * examples/pi.cpp:41-80: neighbours multiplied level by level, an odd tail
 * carried up), each level one set of launches over the whole level; values
 * stay on the GPU.  The device form writes the product zero padded to
 * `width` = the smallest power of two >= n limbs (out_cap >= width) and
 * returns when it is complete; the host form strips leading zeros. */
int bgpu_product_tree_device(const uint64_t* d_leaves, size_t n, uint64_t* d_out, size_t out_cap,
                             void* stream);
int bgpu_product_tree_u64(const uint64_t* leaves, size_t n, uint64_t* out, size_t out_cap,
                          size_t* out_len);

/* Test hook for the products beyond the largest transform (the size range
 * the reference gives to ssa::mul, src/mul/ssa.cpp:383-401 via
 * include/bigint/mul.h:208-220).  Such products cut both operands into blocks
 * of `limbs` u64 limbs and run every block pair as one NTT product; by default
 * the block is 2^24 limbs, whose block pairs fill the largest transform.  A
 * smaller power of two in [64, 2^24] makes every product above 4 * limbs
 * 32-bit points take the block path, so tests can check it against the
 * oracle at small sizes; 0 restores the default. */
int bgpu_set_block_limbs(uint64_t limbs);

/* Transform split used for 2^log2_points-point products: the column pass
 * length 2^log2_column (the row pass gets the rest).  Set by the autotuner
 * (bigint_b200/autotune.py); log2_column = 0 restores the built-in choice.
 * No reference counterpart (the reference has one radix-2 schedule,
 * src/mul/ntt_multithread.cpp:333-379). */
int bgpu_set_split(uint32_t log2_points, uint32_t log2_column);
/* The column length exponent currently used for 2^log2_points points. */
int bgpu_get_split(uint32_t log2_points);
/* The same for the NTT classes of batch plans and product-tree levels, which
 * the autotuner sets for throughput rather than single-product latency. */
int bgpu_set_batch_split(uint32_t log2_points, uint32_t log2_column);
int bgpu_get_batch_split(uint32_t log2_points);

/* Method crossovers used by BGPU_METHOD_AUTO.  They replace the reference's
 * fixed dispatch thresholds (_mul, include/bigint/mul.h:208-220: brute up to
 * 16384 total bits, FFT up to fft::MAX_TOTAL_BITS, NTT above) with values the
 * autotuner measures on the device. */
#define BGPU_TUNE_SCHOOLBOOK_MAX_LIMBS 1u       /* single products: schoolbook for na+nb <= v (<= 256) */
#define BGPU_TUNE_BATCH_SCHOOLBOOK_MAX_LIMBS 2u /* batch plans and tree levels: same, per product */
#define BGPU_TUNE_FFT_MIN_LIMBS 3u              /* host API: FFT form for na+nb in [min, max] ... */
#define BGPU_TUNE_FFT_MAX_LIMBS 4u              /* ... max = 0 disables the FFT form under AUTO */
#define BGPU_TUNE_KARATSUBA_MAX_LIMBS 5u        /* single products: Karatsuba for na+nb <= v (<= 512;
                                                   0 = off), above the schoolbook limit */
#define BGPU_TUNE_BATCH_KARATSUBA_MAX_LIMBS 6u  /* batch plans and tree levels: same */
int bgpu_set_tuning(uint32_t key, uint64_t value);
int bgpu_get_tuning(uint32_t key, uint64_t* value);

/* Apply a tuning table written by the autotuner: a text file, one setting
 * per line ('#' starts a comment):
 *     split <log2_points> <log2_column>    batch_split <log2_points> <log2_column>
 *     schoolbook_max_limbs <n>      batch_schoolbook_max_limbs <n>
 *     karatsuba_max_limbs <n>       batch_karatsuba_max_limbs <n>
 *     fft_min_limbs <n>             fft_max_limbs <n>
 * The whole file is checked before anything is applied; an unknown key or an
 * out-of-range value gives BGPU_ERR_INVALID_ARG and changes nothing. */
int bgpu_load_tuning(const char* path);

/* Largest product of bgpu_mul_u64_device_noalloc: na + nb u64 limbs. */
#define BGPU_NOALLOC_MAX_LIMBS 65536u

/* Device-resident product that allocates nothing.  No counterpart in the
 * reference (its CPU multiply allocates std::vectors freely); it exists for
 * callers that cannot allocate device memory when they multiply: code running
 * inside a fixed memory budget or a caller-managed pool that must not grow,
 * and host threads that may not call cudaMalloc because it can synchronize the
 * whole device.  It runs the same NTT kernels as bgpu_mul_u64_device, with all
 * scratch in one static device array (about 3.8 MB, plus 0.35 MB of static
 * twiddle tables) that every GPU loading this library holds until the process
 * exits; it calls no cudaMalloc, cudaFree or other allocating routine.
 *  - d_a, d_b, d_out are device pointers on the current device; d_out receives
 *    na + nb limbs; d_a == d_b with na == nb squares.
 *  - na + nb must be <= BGPU_NOALLOC_MAX_LIMBS, else BGPU_ERR_CAPACITY and
 *    nothing is launched.
 *  - the first call on each device does the set-up (table upload and the
 *    static array's address, synchronous).
 *  - the call is synchronous: the work is queued on `stream` (0 = legacy
 *    default stream) and the call returns after it completes, with
 *    BGPU_ERR_DEVICE_TIMEOUT if the carry scan's bounded wait gave up.
 *  - every call shares the static array (it keeps the last call's contents;
 *    the carry-scan state is cleared at the start of each call).  Calls in one
 *    process are serialized per device by a host lock held until their work
 *    has finished; work that still overlapped on the GPU would race on the
 *    array. */
int bgpu_mul_u64_device_noalloc(const uint64_t* d_a, size_t na, const uint64_t* d_b, size_t nb,
                                uint64_t* d_out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BIGINT_B200_H */
