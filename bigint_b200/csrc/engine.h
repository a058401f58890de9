// Internal interfaces between the host engine and the CUDA kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "arith.cuh"

namespace bgpu {

// Input/output digit formats on the device.
enum DigitFormat : int {
    kFmtLimb64 = 0,  // little-endian uint64_t limbs (the reference's _mul / ntt::mul seam)
    kFmtDigit28 = 1, // little-endian uint32_t digits of 28 bits (the reference's Digits)
};

// Constants of one prime set, kept in __constant__ memory (one slot per owner
// and prime set) so kernels can index them by the runtime prime number.
struct NttConsts {
    PrimeInfo pr[kNumPrimes];
    uint32_t one_w[kNumPrimes], one_wp[kNumPrimes];  // Montgomery form of 1 (reduces any u32 mod p)
    uint32_t red[kNumPrimes];  // floor(2^32 / p): Shoup form of 1, reduces any u32 into [0, 2p)
    const uint2* stage[kNumPrimes][2];  // [prime][dir] Shoup pairs: entry h+m = omega_{2h}^{+-m}
    const uint2* th[kNumPrimes][2];     // Montgomery pairs: omega_{2^log_max}^{+-(i << split)}
    const uint2* tl[kNumPrimes][2];     // Montgomery pairs: omega_{2^log_max}^{+-i}
    // Garner CRT for p0 < p1 < p2 (Montgomery constants with their w').
    uint32_t k1, k1p;  // p0^-1 mod p1
    uint32_t k2, k2p;  // p0 mod p2
    uint32_t k3, k3p;  // (p0 p1)^-1 mod p2
    uint64_t m01;      // p0 * p1
    int log_max, split;
};

// Constant slots: the engine's two prime sets, then the no-allocation path's.
constexpr int kSlotEngine = 0;   // + prime set
constexpr int kSlotNoAlloc = 2;  // + prime set
constexpr int kConstSlots = 4;
cudaError_t upload_consts(int slot, const NttConsts& c);

// One operand of a transform: a device pointer in `fmt` with `nsrc` source
// elements; `nd32` is its length in 32-bit digits.
struct OperandDesc {
    const void* ptr;
    uint32_t nsrc;
    uint32_t nd32;
    int fmt;
};

// Everything one product needs; the products of one launch share N and
// whether they are squares.
struct ProductDesc {
    OperandDesc op[2];  // op[1] == op[0] when squaring
    uint32_t* y;        // (square ? 1 : 2) * 3 * N residues
    uint64_t* chunks;   // N/2 limbs (8-coefficient chunk sums)
    uint64_t* spill;    // N/8 spills
    uint64_t* flags;    // carry-scan block status words
    void* out;          // output in the launch's format
    size_t out_cap;     // elements of out
};

// Shape of a two-pass transform of N = N1 * N2 points.
struct TransformShape {
    int log_n;   // log2 N
    int log_n1;  // row length (middle pass)
    int log_n2;  // column length (outer passes)
};

// Small products, one CTA each (small_kernels.cu); out has na+nb limbs.
struct SchoolDesc {
    const uint64_t* a;
    const uint64_t* b;
    uint64_t* out;
    uint32_t na, nb;
};
constexpr uint32_t kSchoolbookMaxLimbs = 256;  // schoolbook: na + nb
constexpr uint32_t kKaratsubaMaxLimbs = 256;   // Karatsuba: na and nb each

// Per-launch argument blocks of the NTT passes: a device descriptor array
// for batches, or the single product's descriptor inline (descs == nullptr).
struct FwdColsArgs {
    const ProductDesc* descs;
    ProductDesc one;
    int nops, log_n, log_n1, slot;
    // 1: the operands and this pass's residue planes are free of the
    // preceding kernel (its trigger came after the previous product's
    // inverse pass finished), so the pass starts under that kernel's tail and
    // waits for it only at the end -- which keeps every later kernel ordered
    // after it, since each of them waits for this pass to complete
    int overlap;
};

struct MidRowsArgs {
    const ProductDesc* descs;  // y: A's planes (result in place), then B's unless squaring
    ProductDesc one;
    int log_n, log_n2, slot;
    uint32_t scale_w[kNumPrimes], scale_wp[kNumPrimes];  // N^-1 * 2^32 mod p (Montgomery form)
};

struct InvColsArgs {
    const ProductDesc* descs;  // y (A's planes after the middle pass), chunks, spill
    ProductDesc one;
    int log_n, log_n1, slot;
    uint32_t* err;  // sticky device error word (a bounded wait that gave up), or nullptr
};

// Spectral sums (products beyond the largest transform): the row-pass launch
// that finishes an operand block's forward transform in place (y = its
// spectrum), or the one that forms sum_t sa[t] (.) sb[t] over nterms pairs
// of block spectra and runs the row DIT into y (3 planes each).
constexpr int kMaxSpecTerms = 4;
struct SpecArgs {
    const uint32_t* sa[kMaxSpecTerms];
    const uint32_t* sb[kMaxSpecTerms];
    int nterms;
    uint32_t* y;
    int log_n, log_n2, slot;
    uint32_t scale_w[kNumPrimes], scale_wp[kNumPrimes];  // N^-1 * 2^32 mod p (Montgomery form)
};

// A mixed-length batch (all its NTT classes in one launch per pass): one
// class of products of equal transform length and squaring flag, with its
// CTA range in each pass's launch (begin[3] is its first carry ticket).
struct MixedClass {
    FwdColsArgs fwd;
    MidRowsArgs mid;
    InvColsArgs inv;
    uint32_t begin[4];
    uint32_t tiles, rows, count;  // column tiles (N1 / 8), rows (N2), products
    uint32_t nchunks, bpp;        // carry chunks and carry blocks per product
    uint32_t mid_words;           // shared-memory words of one row in the row pass
    int log_n1, log_n2, square;
};
constexpr int kMaxMixedClasses = 32;
struct MixedArgs {
    const MixedClass* classes;  // device array, in CTA-range order
    int nclasses;
    // each class's first CTA in each pass (carry: first ticket), kept in the
    // launch's parameters so a CTA finds its class from the constant bank
    uint32_t begin[4][kMaxMixedClasses];
    unsigned long long* ticket;  // carry tickets of this launch, from ticket_base
    uint64_t ticket_base;
    uint64_t epoch;
    uint32_t* err;
    // small products of the same batch, one CTA each, after the row pass's
    // CTAs (schoolbook) and the inverse pass's (Karatsuba)
    const SchoolDesc* school;
    uint32_t nschool;
    const SchoolDesc* kara;
    uint32_t nkara;
    uint32_t ntt_blocks[4];  // the NTT CTAs of each pass (small products follow them)
};
struct MixedClassSpec {
    const ProductDesc* descs;  // device descriptors of the class's products
    uint32_t count;
    int log_n;
    bool square;
};
struct MixedSizes {
    uint32_t blocks[4];  // NTT CTAs of each pass's launch (carry: tickets)
    size_t smem[4];      // dynamic shared memory of each launch's NTT CTAs
};
// A class the mixed launches can run (lazy prime set, column tiles of at most
// 2^9 rows, rows of at most 2^9 points, at the batch split).
bool mixed_class_ok(int log_n, bool square);
// Fill the host copy of `nclasses` classes (descs already on the device) and
// the launch sizes; -1 when a class does not qualify.
int mixed_fill(MixedClass* classes, int nclasses, const MixedClassSpec* spec, int slot, const NttConsts& c,
               MixedSizes* sizes);
// The four launches of a mixed-length batch on `stream`.
cudaError_t launch_ntt_mixed(const MixedArgs& m, const MixedSizes& sizes, cudaStream_t stream);

TransformShape choose_shape(int log_n);        // the tuned split (bgpu_set_split), else the built-in one
TransformShape choose_shape_batch(int log_n);  // batch classes (bgpu_set_batch_split), else built-in
TransformShape builtin_shape(int log_n);       // the built-in split only
int set_split(int log_n, int log_n2);  // 0 on success; log_n2 == 0 restores the default
int set_batch_split(int log_n, int log_n2);
bool shape_supported(int log_n, bool square);
bool shape_supported_batch(int log_n, bool square);
size_t smem_fwd_cols(int log_n2, int cols);
size_t smem_mid_rows(int log_n1, bool square);
size_t smem_inv_cols(int log_n2);

// Per-call scratch for one product (device pointers).
struct ProductScratch {
    uint32_t* y;          // (square ? 1 : 2) * 3 * N residues
    uint64_t* chunks;     // N/2 limbs: 8-digit chunk sums before the carry scan
    uint64_t* spill;      // N/8 spills (chunk overflow above 256 bits)
    uint64_t* flags;      // carry-scan block status words
    unsigned long long* ticket;  // carry-scan block ticket counter
    uint32_t* err;        // sticky device error word
};

struct CarryLaunch {
    uint64_t ticket_base;
    uint64_t epoch;
    unsigned long long* ticket = nullptr;  // batch launches: ticket counter
    uint32_t* err = nullptr;               // batch launches: sticky error word
    // The forward pass may run under the tail of whatever kernel precedes it
    // on the stream (the previous product's carry scan), waiting for it only
    // before it exits; only for operands that nothing in flight writes.
    bool overlap_prev = false;
    // Single products: the carry scan in the narrow shape (ticket count
    // carry_blocks_narrow), for a product whose forward pass waited for its
    // predecessor (a chain of dependent products, whose scans overlap nothing).
    bool narrow = false;
};

// Launch the full NTT product pipeline (4 kernels) on `stream`.
// out: device buffer in `out_fmt` with `out_cap` elements.
// `slot` selects the constants (kSlotEngine/kSlotNoAlloc + prime_set_for(log_n));
// `host` is the same constants on the host (for per-call scale factors).
// `ev` (optional) holds 5 events recorded around the 4 launches.  `shape`
// (optional) fixes the split; by default the tuned choice for log_n is used.
cudaError_t launch_ntt_product(int slot, const NttConsts& host, const OperandDesc& a,
                               const OperandDesc& b, bool square, int log_n,
                               const ProductScratch& s, void* out, int out_fmt, size_t out_cap,
                               const CarryLaunch& cl, cudaStream_t stream,
                               cudaEvent_t* ev = nullptr, const TransformShape* shape = nullptr);
constexpr int kNttLaunches = 4;
extern const char* const kNttKernelNames[kNttLaunches];

// Carry-scan blocks: kCarryThreads threads, each resolving kCarryPer
// consecutive 8-coefficient chunks.
#ifndef BGPU_CARRY_THREADS
#define BGPU_CARRY_THREADS 256
#endif
#ifndef BGPU_CARRY_PER
#define BGPU_CARRY_PER 4
#endif
constexpr int kCarryThreads = BGPU_CARRY_THREADS;
constexpr int kCarryPer = BGPU_CARRY_PER;
constexpr uint32_t kCarryChunksPerBlock = (uint32_t)(kCarryThreads * kCarryPer);
uint32_t carry_blocks(uint32_t nchunks);
// The narrow shape, for a single product that waits for its predecessor
// (CarryLaunch::narrow): more, smaller blocks shorten the scan on the
// product's critical path (2^20 points: 66.70 -> 66.15 us per product back to
// back), while a scan that runs under the next product's forward pass keeps
// the default (63.60 against 63.81 us there).  Scratch sized for a product's
// flag words takes the narrow count, the larger of the two.
constexpr int kCarryNarrowThreads = 128;
constexpr int kCarryNarrowPer = 2;
uint32_t carry_blocks_narrow(uint32_t nchunks);

// Diagnostic launch of the carry scan's bounded wait on one flag word.
cudaError_t launch_wait_selftest(const uint64_t* flag, uint64_t epoch, uint32_t limit, uint32_t* err,
                                 cudaStream_t st);

// Batched NTT products: `count` products of 2^log_n points described by the
// device array `descs`, four launches in all (one per pass, a grid slice per
// product); the carry scan takes count * carry_blocks(N/8) tickets.
cudaError_t launch_ntt_batch(int slot, const NttConsts& host, const ProductDesc* descs, int count,
                             bool square, int log_n, int out_fmt, const CarryLaunch& cl,
                             cudaStream_t stream);

// Spectral sums of block products (2 launches per operand block, 3 or 4 per
// sum): spectral_supported(log_n) tells whether the row-pass kernels exist
// for the tuned split of 2^log_n points.  launch_ntt_spectrum writes the
// forward transform of operand `a` (3 planes of 2^log_n residues, in the row
// pass's element order) to `spec`; launch_ntt_spectral_sum multiplies nterms
// pairs of such spectra pointwise, sums them, and inverse-transforms the sum
// through the row DIT and the inverse column pass with CRT; then the sum
// (twice the sum when `twice`) plus the nadd u64 limbs at `add` (nullptr:
// none) is carried into `out_cap` u64 limbs at `out`, which may be the
// limbs at `add` (the doubling is exact limb arithmetic after the CRT).  The
// caller keeps every coefficient of the sum below the product of the three
// primes, and the total below 2^(64 out_cap).
bool spectral_supported(int log_n);
cudaError_t launch_ntt_spectrum(int slot, const NttConsts& host, const OperandDesc& a, int log_n,
                                uint32_t* spec, cudaStream_t stream);
cudaError_t launch_ntt_spectral_sum(int slot, const NttConsts& host, const uint32_t* const* sa,
                                    const uint32_t* const* sb, int nterms, bool twice, int log_n,
                                    const ProductScratch& s, uint64_t* out, size_t out_cap,
                                    const uint64_t* add, size_t nadd, const CarryLaunch& cl,
                                    cudaStream_t stream);

// ---- FP64 complex-FFT form ----
constexpr int kFftMaxLogN = 26;     // largest FFT transform (2^26 complex points)
constexpr int kFftStageLog = 13;    // FFT stage tables cover pair distances < 2^13
constexpr int kFftTwLog = 26, kFftTwSplit = 13;

struct FftConsts {
    const double2* stage[2];  // [dir]: entry h+m = exp(-+ i pi m / h)
    const double2* th[2];     // exp(-+ 2 pi i (i << split) / 2^log_max)
    const double2* tl[2];     // exp(-+ 2 pi i i / 2^log_max)
    int log_max, split;
};
cudaError_t upload_fft_consts(const FftConsts& c);

struct FftShape {
    int log_n, log_n1, log_n2;
};
FftShape fft_choose_shape(int log_n);
bool fft_shape_supported(int log_n);

struct FftScratch {
    double2* y;                  // N complex points
    uint64_t* coef;              // N rounded coefficients
    unsigned long long* maxerr;  // largest |x - round(x)| as double bits
    uint64_t* chunks;            // nchunks * 4 limbs
    uint64_t* spill;             // nchunks
    uint32_t nchunks;            // bits * N / 256
};

// Forward FFT of (A + iB), square, inverse, rounding and chunk sums (4 launches);
// the caller then runs the carry scan over `nchunks` chunks.
cudaError_t launch_fft_product(const uint64_t* a, uint32_t na, const uint64_t* b, uint32_t nb,
                               int bits, int log_n, const FftScratch& s, cudaStream_t stream);
cudaError_t launch_carry(const uint64_t* chunks, const uint64_t* spill, uint32_t nchunks, void* out,
                         int out_fmt, size_t out_cap, const ProductScratch& s, const CarryLaunch& cl,
                         cudaStream_t stream);

// ---- batched products (batch.cu) ----
struct EngineHooks {
    NttConsts consts[kNumSets];
    uint32_t* err;
};
}  // namespace bgpu
struct bgpu_batch_plan_s;
struct bgpu_product;
namespace bgpu {
int batch_plan_create(const bgpu_product* prods, size_t count, uint32_t flags, int device,
                      const EngineHooks& hooks, bgpu_batch_plan_s** out);
int batch_plan_run(bgpu_batch_plan_s* p, cudaStream_t st);
void batch_plan_destroy(bgpu_batch_plan_s* p);
uint32_t batch_plan_launches(const bgpu_batch_plan_s* p);
// Device memory the product tree keeps between calls (grow-only).
struct TreeArena {
    void* ptr = nullptr;
    size_t bytes = 0;
};
// Pairwise product tree of n single-limb values into d_out (width: the
// smallest power of two >= n limbs, zero padded); synchronous on `st`.
int product_tree_device(const uint64_t* d_leaves, size_t n, uint64_t* d_out, size_t out_cap,
                        const EngineHooks& hooks, TreeArena* arena, cudaStream_t st,
                        uint32_t* launches);

cudaError_t launch_schoolbook(const uint64_t* a, uint32_t na, const uint64_t* b, uint32_t nb,
                              uint64_t* out, cudaStream_t stream);
cudaError_t launch_schoolbook_batch(const SchoolDesc* d_descs, uint32_t count, cudaStream_t stream);
cudaError_t launch_karatsuba(const uint64_t* a, uint32_t na, const uint64_t* b, uint32_t nb,
                             uint64_t* out, cudaStream_t stream);
cudaError_t launch_karatsuba_batch(const SchoolDesc* d_descs, uint32_t count, cudaStream_t stream);
inline bool karatsuba_fits(size_t na, size_t nb) { return na <= kKaratsubaMaxLimbs && nb <= kKaratsubaMaxLimbs; }

// Method crossovers, set by the autotuner through bgpu_set_tuning /
// bgpu_load_tuning (defaults below are the built-in choice).
struct Tuning {
    uint32_t schoolbook_max_limbs = kSchoolbookMaxLimbs;        // AUTO single products
    uint32_t batch_schoolbook_max_limbs = kSchoolbookMaxLimbs;  // batch plans and product-tree levels
    uint32_t karatsuba_max_limbs = 0;        // AUTO single products: Karatsuba for na+nb <= this (0 = off)
    uint32_t batch_karatsuba_max_limbs = 0;  // batch plans and product-tree levels (0 = off)
    uint64_t fft_min_limbs = 0, fft_max_limbs = 0;              // AUTO host API: FFT form for na+nb in
                                                                // [min, max]; max 0 = never
};
Tuning& tuning();

// Digit-format conversion kernels (used around the schoolbook path).
cudaError_t launch_digits28_to_limbs(const uint32_t* d, uint32_t nd, uint64_t* limbs,
                                     uint32_t nlimbs, cudaStream_t stream);
cudaError_t launch_limbs_to_digits28(const uint64_t* limbs, uint32_t nlimbs, uint32_t* d,
                                     uint32_t nd, cudaStream_t stream);

// Digit kernels of the device-resident BigFloat steps (bigfloat_kernels.cu).
// A frame operation places operand A at digit offset oa (frame digit j holds
// a[j - oa] when 0 <= j - oa < na, else 0) and B likewise, and writes the L
// frame digits of A + B, or of A - B for A >= B, plus the carry out of the
// frame in out[L].  agg and cin hold frame_blocks(L) words each.
struct FrameOp {
    const uint32_t* a;
    int64_t oa;
    uint32_t na;
    const uint32_t* b;
    int64_t ob;
    uint32_t nb;
    uint32_t L;
    int sub;
    const unsigned long long* order;  // nullptr, or a compare result: B - A when B is larger
};
uint32_t frame_blocks(uint32_t L);
cudaError_t launch_frame_addsub(const FrameOp& f, uint32_t* agg, uint32_t* cin, uint32_t* out,
                                cudaStream_t st);
// Into a zeroed word: (j + 1) << 2 | (1 if A_j > B_j else 2) for the highest
// frame position j where A and B differ; stays 0 when they are equal.
cudaError_t launch_frame_cmp(const FrameOp& f, unsigned long long* r, cudaStream_t st);
// Into three zeroed words: r[0] = (j + 1) << 32 | d[j] for the highest nonzero
// j; r[1], r[2] = 2^32 - j for the lowest nonzero j >= from0, from1 (0: none).
cudaError_t launch_extent(const uint32_t* d, uint32_t n, uint32_t from0, uint32_t from1,
                          unsigned long long* r, cudaStream_t st);
// out = v >> s (n digits) or v << s (n + 1 digits), s in [1, 27], 28-bit digits
cudaError_t launch_shift_digits(const uint32_t* v, uint32_t n, uint32_t s, bool left, uint32_t* out,
                                cudaStream_t st);

// Limb accumulation (huge.cu): out[0..L) += add[0..nadd) (nadd <= L) with the
// carry carried through all of out; agg and cin hold accumulate_blocks(L)
// words each (the pairwise block products' fallback and the decimal
// conversions).  kHugeBlockLimbs is the operand block of products beyond the
// largest transform: a pair of blocks fills the largest NTT transform.
constexpr uint64_t kHugeBlockLimbs = (uint64_t)1 << 24;
// Limbs per leaf of the decimal printer: one thread prints a leaf by repeated
// division by 10^9, its work growing with the square of the leaf.
constexpr uint32_t kPrintLeafLimbs = 32;
// Limbs per leaf of the decimal parser: one thread builds a leaf from its
// decimal digits by Horner's rule, its work growing with the square of the leaf.
constexpr uint32_t kParseLeafLimbs = 32;
uint32_t accumulate_blocks(uint64_t L);
cudaError_t launch_accumulate(uint64_t* out, uint64_t L, const uint64_t* add, uint64_t nadd, uint32_t* agg,
                              uint32_t* cin, cudaStream_t st);

// Decimal text to binary (decimal.cu): leaves of 19 digits built w limbs per
// segment (w <= 128) from dig[0..D) (values 0..9, most significant first), and
// out[p*2w1 ..] += prev[2p*w1 .. 2p*w1 + w1) over nseg segments of 2*w1 limbs.
cudaError_t launch_dec_leaves(const uint8_t* dig, uint64_t D, uint32_t w, uint64_t nseg, uint64_t* out,
                              cudaStream_t st);
cudaError_t launch_seg_add_low(uint64_t* out, const uint64_t* prev, uint32_t w1, uint64_t nseg,
                               cudaStream_t st);

// Binary to decimal (decimal.cu): one block per level-above segment of 2w
// limbs, r = s - U and the one-step quotient correction, written as the two
// w-limb halves of the level below; the decimal text of w-limb leaves; the
// complement r = ~x over el limbs (r[el] = 0); and one exact correction step
// of a reciprocal (r >= q: r -= q, v += 1, *flag = 1).
cudaError_t launch_seg_divstep(const uint64_t* cur, uint64_t* u, uint64_t* t, uint32_t tstride, const uint64_t* q_pow,
                               uint32_t w, uint64_t nseg, uint64_t* next, cudaStream_t st);
cudaError_t launch_dec_print_leaves(const uint64_t* in, uint32_t w, uint64_t nseg, char* out, cudaStream_t st);
cudaError_t launch_not_limbs(const uint64_t* x, uint32_t el, uint64_t* r, cudaStream_t st);
cudaError_t launch_fix_step(uint64_t* r, uint32_t nr, const uint64_t* q, uint32_t nq, uint64_t* v, uint32_t nv,
                            uint32_t* flag, cudaStream_t st);

// Host <-> device copies of the host API: page-locked caller memory goes
// straight to the copy engines, pageable memory through a ring of
// page-locked slots filled by a pool of host threads.  host_to_device may
// return before the copy has finished: a page-locked source must stay
// unchanged until the stream has passed the copy, a pageable one is free at
// once.  With digits_ok it also checks that every 32-bit word is below 2^28.
// device_to_host returns once the bytes are in dst.
int host_to_device(void* dst, const void* src, size_t bytes, cudaStream_t st, bool* digits_ok);
int device_to_host(void* dst, const void* src, size_t bytes, cudaStream_t st);
void release_host_staging();

}  // namespace bgpu
