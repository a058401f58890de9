// Host engine and C-ABI of bigint_b200.
//
// Owns the device, the twiddle tables, a grow-only scratch arena and the
// stream; maps the reference's multiply seams onto the kernel pipelines:
//   bgpu_mul_u64     <- bigint::mul::_mul / ntt::mul   (include/bigint/mul.h:208-220,
//                                                       src/mul/ntt_multithread.cpp:444-530)
//   bgpu_mul_digits  <- bigint::mul::mul_digits        (include/bigint/mul.h:223-318)
//   bgpu_reciprocal_digits <- BigFloat::reciprocal      (src/bigint.cpp:1044-1071)
//   bgpu_divmod_digits     <- BigInt::divmod            (src/bigint.cpp:625-673)
//   bgpu_bigfloat_to_decimal <- BigFloat::print         (src/bigint.cpp:972-1041)
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/bigint_b200.h"
#include "engine.h"
#include "tables.h"

namespace bgpu {
namespace {

struct Engine {
    int device = -1;
    cudaStream_t stream = nullptr;
    // copy streams, slot buffers and events of the pipelined host API
    cudaStream_t h2d = nullptr, d2h = nullptr;
    void* d_many = nullptr;
    size_t many_bytes = 0;
    cudaEvent_t ev_in[4] = {}, ev_comp[4] = {}, ev_out[4] = {};
    NttConsts consts[kNumSets]{};
    void* d_tables[kNumSets] = {};
    void* d_fft_tables = nullptr;
    unsigned long long* d_fft_err = nullptr;
    // scratch arena
    void* d_scratch = nullptr;
    size_t scratch_bytes = 0;
    // small fixed state
    uint32_t* d_err = nullptr;
    unsigned long long* d_ticket = nullptr;
    uint64_t ticket_base = 0, epoch = 0;
    // device I/O buffers of the host API
    void* d_io = nullptr;
    size_t io_bytes = 0;
    TreeArena tree;  // product-tree values, descriptors and scratch
    // digit buffers of the device-resident reciprocal (one per live value)
    uint32_t* rs[23] = {};
    size_t rs_bytes[23] = {};
    // block products of the decomposition beyond the largest transform
    void* d_huge = nullptr;
    size_t huge_bytes = 0;
    // decimal conversion: digits, two level arrays, powers of ten, output
    void* d_dec = nullptr;
    size_t dec_bytes = 0;
    void* d_desc = nullptr;  // small-product descriptors of the decimal levels
    size_t desc_bytes = 0;
    unsigned long long* h_small = nullptr;  // page-locked readback words of the step-by-step paths
    // powers of ten Q_k = 10^(19 * 2^k) (limb 2^k - 1, 2^k limbs) and their
    // reciprocals V_k = floor(2^(128 * 2^k) / Q_k), cached across decimal calls
    uint64_t* d_pq = nullptr;
    size_t pq_bytes = 0;
    int pq_levels = 0;
    uint64_t* d_pv = nullptr;
    size_t pv_bytes = 0;
    int pv_levels = 0;
    // stream and scratch layout of the last NTT product launched
    cudaStream_t ntt_stream = nullptr;
    int ntt_log_n = -1;
    bool ntt_square = false;
    // output of the previous bgpu_mul_u64_device call and its stream
    cudaStream_t prev_stream = nullptr;
    const void* prev_out = nullptr;
    size_t prev_out_bytes = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    uint32_t last_launches = 0;
    // optional per-kernel timing of NTT products: a ring of event sets, one
    // set per product, read back (and averaged) without per-product syncs
    bool kernel_timing = false;
    std::vector<cudaEvent_t> kev;  // kTimingRing * (kNttLaunches + 1)
    uint64_t kev_count = 0;
    // operand block of products beyond the largest transform (a power of
    // two; kHugeBlockLimbs unless a test shrinks it with bgpu_set_block_limbs)
    uint64_t huge_block = kHugeBlockLimbs;
};

constexpr uint64_t kTimingRing = 1024;  // products whose kernel times are kept

Engine g;
std::mutex g_mu;
Tuning g_tuning;

int cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return BGPU_OK;
    if (e == cudaErrorMemoryAllocation) return BGPU_ERR_OOM;
    return BGPU_ERR_CUDA;
}

void release_locked() {
    if (g.device < 0) return;
    cudaSetDevice(g.device);
    if (g.stream) cudaStreamSynchronize(g.stream);
    release_host_staging();
    for (auto t : g.d_tables) cudaFree(t);
    cudaFree(g.d_fft_tables);
    cudaFree(g.d_fft_err);
    cudaFree(g.d_scratch);
    cudaFree(g.d_huge);
    cudaFree(g.d_dec);
    cudaFree(g.d_desc);
    if (g.h_small) cudaFreeHost(g.h_small);
    cudaFree(g.d_pq);
    cudaFree(g.d_pv);
    cudaFree(g.d_err);
    cudaFree(g.d_ticket);
    cudaFree(g.d_io);
    cudaFree(g.tree.ptr);
    for (auto p : g.rs) cudaFree(p);
    if (g.ev0) cudaEventDestroy(g.ev0);
    if (g.ev1) cudaEventDestroy(g.ev1);
    for (auto e : g.kev) cudaEventDestroy(e);
    cudaFree(g.d_many);
    for (int i = 0; i < 4; ++i) {
        if (g.ev_in[i]) cudaEventDestroy(g.ev_in[i]);
        if (g.ev_comp[i]) cudaEventDestroy(g.ev_comp[i]);
        if (g.ev_out[i]) cudaEventDestroy(g.ev_out[i]);
    }
    if (g.h2d) cudaStreamDestroy(g.h2d);
    if (g.d2h) cudaStreamDestroy(g.d2h);
    if (g.stream) cudaStreamDestroy(g.stream);
    g = Engine{};
}

int build_tables_locked() {
    for (int ps = 0; ps < kNumSets; ++ps) {
        std::vector<uint2> host(table_entries(ps, kMaxLogRow));
        build_tables(ps, kMaxLogRow, host.data());
        cudaError_t e = cudaMalloc(&g.d_tables[ps], host.size() * sizeof(uint2));
        if (e != cudaSuccess) return cuda_status(e);
        e = cudaMemcpy(g.d_tables[ps], host.data(), host.size() * sizeof(uint2),
                       cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_status(e);
        g.consts[ps] = make_consts(ps, kMaxLogRow, static_cast<const uint2*>(g.d_tables[ps]));
        e = upload_consts(kSlotEngine + ps, g.consts[ps]);
        if (e != cudaSuccess) return cuda_status(e);
    }
    std::vector<double2> fh(2 * fft_table_block());
    build_fft_tables(fh.data());
    cudaError_t e = cudaMalloc(&g.d_fft_tables, fh.size() * sizeof(double2));
    if (e == cudaSuccess)
        e = cudaMemcpy(g.d_fft_tables, fh.data(), fh.size() * sizeof(double2), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = upload_fft_consts(make_fft_consts(static_cast<const double2*>(g.d_fft_tables)));
    if (e == cudaSuccess) e = cudaMalloc(&g.d_fft_err, sizeof(unsigned long long));
    return cuda_status(e);
}

int init_locked(int device) {
    if (g.device == device) return BGPU_OK;
    release_locked();
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= device || device < 0) return BGPU_ERR_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess) return BGPU_ERR_NO_DEVICE;
    g.device = device;
    int rc = build_tables_locked();
    if (rc == BGPU_OK) rc = cuda_status(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
    if (rc == BGPU_OK) rc = cuda_status(cudaStreamCreateWithFlags(&g.h2d, cudaStreamNonBlocking));
    if (rc == BGPU_OK) rc = cuda_status(cudaStreamCreateWithFlags(&g.d2h, cudaStreamNonBlocking));
    for (int i = 0; i < 4 && rc == BGPU_OK; ++i) {
        rc = cuda_status(cudaEventCreateWithFlags(&g.ev_in[i], cudaEventDisableTiming));
        if (rc == BGPU_OK) rc = cuda_status(cudaEventCreateWithFlags(&g.ev_comp[i], cudaEventDisableTiming));
        if (rc == BGPU_OK) rc = cuda_status(cudaEventCreateWithFlags(&g.ev_out[i], cudaEventDisableTiming));
    }
    if (rc == BGPU_OK) rc = cuda_status(cudaMalloc(&g.d_err, sizeof(uint32_t)));
    if (rc == BGPU_OK) rc = cuda_status(cudaMemset(g.d_err, 0, sizeof(uint32_t)));
    if (rc == BGPU_OK) rc = cuda_status(cudaMalloc(&g.d_ticket, sizeof(unsigned long long)));
    if (rc == BGPU_OK) rc = cuda_status(cudaMemset(g.d_ticket, 0, sizeof(unsigned long long)));
    if (rc == BGPU_OK) rc = cuda_status(cudaEventCreate(&g.ev0));
    if (rc == BGPU_OK) rc = cuda_status(cudaEventCreate(&g.ev1));
    if (rc != BGPU_OK) {
        release_locked();
        return rc == BGPU_ERR_CUDA ? BGPU_ERR_NO_DEVICE : rc;
    }
    return BGPU_OK;
}

int ensure(void** ptr, size_t* have, size_t need) {
    if (*have >= need) return BGPU_OK;
    if (*ptr) {
        cudaStreamSynchronize(g.stream);
        cudaFree(*ptr);
        *ptr = nullptr;
        *have = 0;
    }
    size_t sz = need + need / 4;
    cudaError_t e = cudaMalloc(ptr, sz);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *ptr = nullptr;
        return BGPU_ERR_OOM;
    }
    *have = sz;
    return BGPU_OK;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

int ceil_log2(uint64_t x) {
    int l = 0;
    while (((uint64_t)1 << l) < x) ++l;
    return l;
}

// Scratch for an NTT product of 2^log_n points.
int prepare_scratch(int log_n, bool square, ProductScratch* s) {
    const size_t nn = (size_t)1 << log_n;
    const size_t y_bytes = align256((square ? 1 : 2) * (size_t)kNumPrimes * nn * 4);
    const size_t ch_bytes = align256(nn / 2 * 8);
    const size_t sp_bytes = align256(nn / 8 * 8);
    const size_t fl_bytes = align256((size_t)carry_blocks_narrow((uint32_t)(nn / 8)) * 8);  // either shape
    int rc = ensure(&g.d_scratch, &g.scratch_bytes, y_bytes + ch_bytes + sp_bytes + fl_bytes);
    if (rc != BGPU_OK) return rc;
    char* b = static_cast<char*>(g.d_scratch);
    s->y = reinterpret_cast<uint32_t*>(b);
    s->chunks = reinterpret_cast<uint64_t*>(b + y_bytes);
    s->spill = reinterpret_cast<uint64_t*>(b + y_bytes + ch_bytes);
    s->flags = reinterpret_cast<uint64_t*>(b + y_bytes + ch_bytes + sp_bytes);
    s->ticket = g.d_ticket;
    s->err = g.d_err;
    return BGPU_OK;
}

// Core: product of two device operands into a device output (async).
// nd32 values are operand lengths in 32-bit digits.
int multiply_device(const OperandDesc& a, const OperandDesc& b, bool square, void* out,
                    int out_fmt, size_t out_cap, uint32_t flags, cudaStream_t st,
                    bgpu_stats* stats, bool overlap_prev = false) {
    const uint32_t method = flags & BGPU_METHOD_MASK;
    const uint64_t total32 = (uint64_t)a.nd32 + b.nd32;
    const int log_n = ceil_log2(total32 - 1);
    if (log_n > kMaxLogN || !shape_supported(log_n < 5 ? 5 : log_n, square))
        return BGPU_ERR_CAPACITY;
    const int ln = log_n < 5 ? 5 : log_n;
    ProductScratch s{};
    int rc = prepare_scratch(ln, square, &s);
    if (rc != BGPU_OK) return rc;
    CarryLaunch cl;
    cl.ticket_base = g.ticket_base;
    cl.epoch = ++g.epoch;
    // The scratch layout (residue planes first, then the chunk sums, spills
    // and flags the carry scan reads) depends on the length and on squaring:
    // only an identical layout keeps this forward pass's planes clear of the
    // previous product's carry data while that scan still runs.
    cl.overlap_prev = overlap_prev && st == g.ntt_stream && ln == g.ntt_log_n && square == g.ntt_square;
    cl.narrow = !cl.overlap_prev;
    g.ntt_stream = st;
    g.ntt_log_n = ln;
    g.ntt_square = square;
    const uint32_t nch = (uint32_t)(((size_t)1 << ln) / 8);
    g.ticket_base += cl.narrow ? carry_blocks_narrow(nch) : carry_blocks(nch);
    cudaEvent_t* ev = nullptr;
    if (g.kernel_timing) {
        ev = g.kev.data() + (g.kev_count % kTimingRing) * (kNttLaunches + 1);
        ++g.kev_count;
    }
    const int ps = prime_set_for(ln);
    cudaError_t e = launch_ntt_product(kSlotEngine + ps, g.consts[ps], a, b, square, ln, s, out,
                                       out_fmt, out_cap, cl, st, ev);
    g.last_launches = kNttLaunches;
    if (stats) {
        stats->method = BGPU_METHOD_NTT;
        stats->log2_points = (uint32_t)ln;
    }
    (void)method;
    return cuda_status(e);
}

// True when a product of na x nb limbs needs more points than the largest
// transform.
// Largest transform a single product uses: a block pair of huge_block limbs
// each fills 2^(log2(huge_block) + 2) points, exactly the largest transform
// for the default block.
int transform_cap_log() { return ceil_log2(g.huge_block) + 2; }

bool beyond_transform(size_t na, size_t nb) {
    return ceil_log2(2 * (uint64_t)(na + nb) - 1) > transform_cap_log();
}

// Largest number of block products one spectral sum may hold: a block has at
// most 2S 32-bit digits, so a block product's coefficients are below
// 2S (2^32 - 1)^2, and the sum's must stay below the product of the three
// primes for the CRT to return them exactly.  2 for the default 2^24-limb
// blocks (2^90 against 2^90.47).
int spectral_terms(int ps, uint64_t S) {
    const PrimeSetInfo& s = kPrimeSets[ps];
    const unsigned __int128 m = (unsigned __int128)s.p[0] * s.p[1] * s.p[2];
    const unsigned __int128 per = (unsigned __int128)0xFFFFFFFFu * 0xFFFFFFFFu * (2 * S);
    const unsigned __int128 t = (m - 1) / per;
    return (int)(t < (unsigned __int128)kMaxSpecTerms ? t : kMaxSpecTerms);
}

// The spectral form of a product beyond the largest transform:
//   A * B = sum_k 2^(64 S k) C_k,  C_k = sum_{i+j=k} A_i B_j,
// with every block's transform computed once (its spectrum, 3 N residues)
// and each C_k formed in the transform domain as sums of at most `tmax`
// pointwise products.  Each sum is inverse-transformed once (row DIT,
// inverse column pass with CRT) and carried straight into dout's window of
// 2S + 1 limbs at offset S k, together with what that window already holds
// (the chunk merge before the carry scan).  Output blocks go in increasing
// k, so above limb (k+1)S + 1 dout is still zero when C_k's first sum
// arrives, and every partial sum of the product that ends with (part of)
// C_k is below 2^(64 (kS + 2S + 1)): nothing carries out of the window.  A
// square's off-diagonal pairs (i < j) are summed once and doubled in the
// merge, its diagonal squares summed on their own.  The pairwise form
// multiplies every block pair as a whole product: 3 transforms per pair
// against about 1 here.
int huge_spectral(const uint64_t* da, size_t na, const uint64_t* db, size_t nb, uint64_t* dout, bool square,
                  int tmax, cudaStream_t st) {
    const uint64_t S = g.huge_block, L = na + nb;
    const int ln = transform_cap_log(), ps = prime_set_for(ln);
    const size_t nn = (size_t)1 << ln;
    const uint64_t nA = (na + S - 1) / S, nB = square ? nA : (nb + S - 1) / S;
    const size_t nspec = nA + (square ? 0 : nB);
    const size_t spec_bytes = align256((size_t)kNumPrimes * nn * 4);
    int rc = ensure(&g.d_huge, &g.huge_bytes, nspec * spec_bytes);
    if (rc != BGPU_OK) return rc;
    char* base = static_cast<char*>(g.d_huge);
    auto spec = [&](uint64_t i) { return reinterpret_cast<uint32_t*>(base + i * spec_bytes); };
    ProductScratch s{};
    rc = prepare_scratch(ln, true, &s);  // 3 residue planes: the sums' row pass output
    if (rc != BGPU_OK) return rc;
    const int slot = kSlotEngine + ps;
    cudaError_t e = cudaMemsetAsync(dout, 0, L * 8, st);
    for (uint64_t i = 0; e == cudaSuccess && i < nspec; ++i) {
        const bool from_a = i < nA;
        const uint64_t off = (from_a ? i : i - nA) * S;
        const uint64_t len = std::min<uint64_t>(S, (from_a ? na : nb) - off);
        const OperandDesc od{(from_a ? da : db) + off, (uint32_t)len, (uint32_t)(2 * len), kFmtLimb64};
        e = launch_ntt_spectrum(slot, g.consts[ps], od, ln, spec(i), st);
    }
    if (e != cudaSuccess) return cuda_status(e);
    // (i, j) pairs of output block k in sums of at most tmax; `first`: the
    // window holds only C_(k-1)'s top S + 1 limbs so far (nothing when k = 0)
    auto run_sums = [&](const std::vector<std::pair<uint64_t, uint64_t>>& pairs, uint64_t k, bool twice,
                        bool& first) {
        const uint64_t off = k * S, win = std::min<uint64_t>(2 * S + 1, L - off);
        for (size_t g0 = 0; g0 < pairs.size(); g0 += (size_t)tmax) {
            const int n = (int)std::min<size_t>((size_t)tmax, pairs.size() - g0);
            const uint32_t* sa[kMaxSpecTerms];
            const uint32_t* sb[kMaxSpecTerms];
            for (int t = 0; t < n; ++t) {
                sa[t] = spec(pairs[g0 + t].first);
                sb[t] = spec(square ? pairs[g0 + t].second : nA + pairs[g0 + t].second);
            }
            const uint64_t nadd = first ? (k == 0 ? 0 : std::min<uint64_t>(S + 1, win)) : win;
            first = false;
            CarryLaunch cl;
            cl.ticket_base = g.ticket_base;
            cl.epoch = ++g.epoch;
            g.ticket_base += carry_blocks((uint32_t)(nn / 8));
            const cudaError_t e2 = launch_ntt_spectral_sum(slot, g.consts[ps], sa, sb, n, twice, ln, s, dout + off,
                                                           win, nadd ? dout + off : nullptr, nadd, cl, st);
            if (e2 != cudaSuccess) return e2;
        }
        return cudaSuccess;
    };
    std::vector<std::pair<uint64_t, uint64_t>> once, twice;
    for (uint64_t k = 0; e == cudaSuccess && k + 1 < nA + nB; ++k) {
        once.clear();
        twice.clear();
        for (uint64_t i = k >= nB ? k - (nB - 1) : 0; i <= k && i < nA; ++i) {
            const uint64_t j = k - i;
            if (!square)
                once.emplace_back(i, j);
            else if (i < j)
                twice.emplace_back(i, j);
            else if (i == j)
                once.emplace_back(i, j);
        }
        bool first = true;
        e = run_sums(once, k, false, first);
        if (e == cudaSuccess) e = run_sums(twice, k, true, first);
    }
    g.ntt_log_n = -1;  // no forward pass overlaps the carry scans that end this product
    return cuda_status(e);
}

// Product beyond the largest transform (huge.cu): both operands in blocks of
// g.huge_block limbs (2^24: 2^30 bits) added into dout (na + nb limbs) at
// their offsets with a carry scan over the rest.  The spectral form
// (huge_spectral) when its row kernels exist for the block's transform and its
// spectra fit in device memory; otherwise every block pair is one NTT
// product, a square computing each off-diagonal pair once and adding it
// twice.
int huge_product(const uint64_t* da, size_t na, const uint64_t* db, size_t nb, uint64_t* dout, bool square,
                 cudaStream_t st) {
    const int ln = transform_cap_log();
    const int tmax = spectral_terms(prime_set_for(ln), g.huge_block);
    if (tmax >= 1 && spectral_supported(ln)) {
        const int rc = huge_spectral(da, na, db, nb, dout, square, tmax, st);
        if (rc != BGPU_ERR_OOM) return rc;
    }
    const uint64_t S = g.huge_block, L = na + nb;
    const size_t acc = align256((size_t)accumulate_blocks(L) * 4);
    int rc = ensure(&g.d_huge, &g.huge_bytes, 2 * S * 8 + 2 * acc);
    if (rc != BGPU_OK) return rc;
    uint64_t* tmp = static_cast<uint64_t*>(g.d_huge);
    uint32_t* agg = reinterpret_cast<uint32_t*>(reinterpret_cast<char*>(g.d_huge) + 2 * S * 8);
    uint32_t* cin = reinterpret_cast<uint32_t*>(reinterpret_cast<char*>(agg) + acc);
    cudaError_t e = cudaMemsetAsync(dout, 0, L * 8, st);
    if (e != cudaSuccess) return cuda_status(e);
    for (uint64_t ia = 0; ia < na; ia += S) {
        for (uint64_t ib = square ? ia : 0; ib < nb; ib += S) {
            const uint64_t la = std::min<uint64_t>(S, na - ia), lb = std::min<uint64_t>(S, nb - ib);
            const bool diag = square && ia == ib;
            OperandDesc oa{da + ia, (uint32_t)la, (uint32_t)(2 * la), kFmtLimb64};
            OperandDesc ob{db + ib, (uint32_t)lb, (uint32_t)(2 * lb), kFmtLimb64};
            rc = multiply_device(oa, diag ? oa : ob, diag, tmp, kFmtLimb64, la + lb, BGPU_METHOD_AUTO, st,
                                 nullptr);
            if (rc != BGPU_OK) return rc;
            for (int twice = 0; twice < (square && !diag ? 2 : 1); ++twice) {
                e = launch_accumulate(dout + ia + ib, L - (ia + ib), tmp, la + lb, agg, cin, st);
                if (e != cudaSuccess) return cuda_status(e);
            }
        }
    }
    return BGPU_OK;
}

// The small-product kernel a call uses (BGPU_METHOD_AUTO: by the tuned
// crossovers), or 0 for the transform methods.
uint32_t small_method(uint32_t flags, size_t na, size_t nb) {
    const uint32_t m = flags & BGPU_METHOD_MASK;
    if (m == BGPU_METHOD_SCHOOLBOOK || m == BGPU_METHOD_KARATSUBA) return m;
    if (m != BGPU_METHOD_AUTO) return 0;
    const Tuning& t = tuning();
    if (na + nb <= t.schoolbook_max_limbs) return BGPU_METHOD_SCHOOLBOOK;
    if (na + nb <= t.karatsuba_max_limbs && karatsuba_fits(na, nb)) return BGPU_METHOD_KARATSUBA;
    return 0;
}

// Launch the small-product kernel `m` (schoolbook or Karatsuba); operands
// beyond the kernel's limits are an invalid argument.
int launch_small(uint32_t m, const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out,
                 cudaStream_t st) {
    if (m == BGPU_METHOD_SCHOOLBOOK) {
        if (na + nb > kSchoolbookMaxLimbs) return BGPU_ERR_INVALID_ARG;
        return cuda_status(launch_schoolbook(a, (uint32_t)na, b, (uint32_t)nb, out, st));
    }
    if (!karatsuba_fits(na, nb)) return BGPU_ERR_INVALID_ARG;
    return cuda_status(launch_karatsuba(a, (uint32_t)na, b, (uint32_t)nb, out, st));
}

bool valid_method(uint32_t flags, bool allow_fft) {
    const uint32_t m = flags & BGPU_METHOD_MASK;
    return m == BGPU_METHOD_AUTO || m == BGPU_METHOD_NTT || m == BGPU_METHOD_SCHOOLBOOK ||
           m == BGPU_METHOD_KARATSUBA || (allow_fft && m == BGPU_METHOD_FFT);
}

// AUTO picks the FFT form only inside the tuned limb range.
bool auto_fft(uint32_t flags, size_t na, size_t nb) {
    if ((flags & BGPU_METHOD_MASK) != BGPU_METHOD_AUTO) return false;
    const Tuning& t = tuning();
    return t.fft_max_limbs != 0 && na + nb >= t.fft_min_limbs && na + nb <= t.fft_max_limbs;
}

constexpr double kFftMaxErr = 0.25;  // larger rounding distances are recomputed on the NTT

unsigned long long* small_host();

int check_device_error(int rc) {
    if (rc != BGPU_OK) return rc;
    uint32_t err = 0;
    unsigned long long* hp = small_host();  // page-locked: no driver staging pass
    uint32_t* dst = hp ? reinterpret_cast<uint32_t*>(hp + 7) : &err;
    cudaError_t e = cudaMemcpyAsync(dst, g.d_err, sizeof(err), cudaMemcpyDeviceToHost, g.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g.stream);
    if (e != cudaSuccess) return cuda_status(e);
    err = *dst;
    if (err) {
        // Clear the error and restart the carry-scan tickets from zero, so a
        // launch that failed part-way cannot leave the counter and the host's
        // ticket base out of step for the next product.
        cudaMemsetAsync(g.d_err, 0, sizeof(uint32_t), g.stream);
        cudaMemsetAsync(g.d_ticket, 0, sizeof(unsigned long long), g.stream);
        cudaStreamSynchronize(g.stream);
        g.ticket_base = 0;
        return BGPU_ERR_DEVICE_TIMEOUT;
    }
    return BGPU_OK;
}

size_t strip64(const uint64_t* x, size_t n) {
    while (n > 0 && x[n - 1] == 0) --n;
    return n;
}

size_t strip32(const uint32_t* x, size_t n) {
    while (n > 0 && x[n - 1] == 0) --n;
    return n;
}

// Bit length of n >= 1 28-bit digits whose top digit is nonzero.
uint64_t bits28(const uint32_t* d, size_t n) {
    return 28 * (uint64_t)(n - 1) + (32 - __builtin_clz(d[n - 1]));
}

// Bits per FFT point.  Worst-case mode: the largest b in [8, 20] with
//   2b <= 46 - L - log2(L + 1),   L = log2 of the transform length,
// which keeps the error of every coefficient below 1/4 by Percival's bound for
// FFT convolution (Math. Comp. 72 (2003), Thm. 5.1) applied to x = A + iB,
// ||x||^2 <= 2N(2^b - 1)^2, with one extra complex multiply per point for the
// two-pass twiddle and a one-bit margin.  Average mode (BGPU_FFT_AVERAGE_BOUND):
//   2b <= 50 - L/2 - log2(L + 1),
// the random-walk growth of the error; products whose measured error exceeds
// 1/4 are recomputed on the NTT.  Both modes also keep every coefficient below
// 2^49 so its rounding distance is meaningful.
int fft_pick(size_t na, size_t nb, uint32_t flags, int* bits, int* log_n) {
    const int forced = (int)((flags >> 8) & 0x1Fu);
    const bool avg = (flags & BGPU_FFT_AVERAGE_BOUND) != 0;
    for (int b = forced ? forced : 20; b >= (forced ? forced : 8); --b) {
        const uint64_t npa = (na * 64 + b - 1) / b, npb = (nb * 64 + b - 1) / b;
        int L = 0;
        while (((uint64_t)1 << L) < npa + npb - 1) ++L;
        if (L < 8) L = 8;
        if (!fft_shape_supported(L)) continue;
        const double lim = avg ? 50.0 - L / 2.0 - std::log2(L + 1.0) : 46.0 - L - std::log2(L + 1.0);
        if (!forced && 2.0 * b > lim) continue;
        // coefficients (< min(npa, npb) * 2^2b) must stay below 2^49, where the
        // rounding distance can still certify them (doubles are 1/16 apart)
        if (!forced && 2.0 * b + std::log2((double)std::min(npa, npb)) > 49.0) continue;
        *bits = b;
        *log_n = L;
        return BGPU_OK;
    }
    return BGPU_ERR_CAPACITY;
}

// FFT product into dout (na + nb limbs); returns the measured max error.
int fft_product_locked(const uint64_t* da, size_t na, const uint64_t* db, size_t nb, int bits,
                       int log_n, uint64_t* dout, cudaStream_t st, double* maxerr) {
    const size_t nn = (size_t)1 << log_n;
    const uint32_t nchunks = (uint32_t)((uint64_t)bits * nn / 256);
    const size_t y_bytes = align256(nn * sizeof(double2)), co_bytes = align256(nn * 8);
    const size_t ch_bytes = align256((size_t)nchunks * 32), sp_bytes = align256((size_t)nchunks * 8);
    const size_t fl_bytes = align256((size_t)carry_blocks(nchunks) * 8);
    int rc = ensure(&g.d_scratch, &g.scratch_bytes, y_bytes + co_bytes + ch_bytes + sp_bytes + fl_bytes);
    if (rc != BGPU_OK) return rc;
    char* base = static_cast<char*>(g.d_scratch);
    FftScratch fs{};
    fs.y = reinterpret_cast<double2*>(base);
    fs.coef = reinterpret_cast<uint64_t*>(base + y_bytes);
    fs.chunks = reinterpret_cast<uint64_t*>(base + y_bytes + co_bytes);
    fs.spill = reinterpret_cast<uint64_t*>(base + y_bytes + co_bytes + ch_bytes);
    fs.maxerr = g.d_fft_err;
    fs.nchunks = nchunks;
    ProductScratch ps{};
    ps.flags = reinterpret_cast<uint64_t*>(base + y_bytes + co_bytes + ch_bytes + sp_bytes);
    ps.ticket = g.d_ticket;
    ps.err = g.d_err;
    cudaError_t e = cudaMemsetAsync(g.d_fft_err, 0, sizeof(unsigned long long), st);
    if (e == cudaSuccess) e = launch_fft_product(da, (uint32_t)na, db, (uint32_t)nb, bits, log_n, fs, st);
    if (e != cudaSuccess) return cuda_status(e);
    CarryLaunch cl;
    cl.ticket_base = g.ticket_base;
    cl.epoch = ++g.epoch;
    g.ticket_base += carry_blocks(nchunks);
    e = launch_carry(fs.chunks, fs.spill, nchunks, dout, kFmtLimb64, na + nb, ps, cl, st);
    if (e != cudaSuccess) return cuda_status(e);
    g.last_launches = 5;
    unsigned long long bitsv = 0;
    e = cudaMemcpyAsync(&bitsv, g.d_fft_err, sizeof(bitsv), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_status(e);
    memcpy(maxerr, &bitsv, sizeof(double));
    return BGPU_OK;
}

int mul_u64_locked(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out,
                   size_t out_cap, size_t* out_len, uint32_t flags, bgpu_stats* stats) {
    const bool square = (a == b && na == nb);
    na = strip64(a, na);
    nb = square ? na : strip64(b, nb);
    if (stats) memset(stats, 0, sizeof(*stats));
    if (na == 0 || nb == 0) {
        *out_len = 0;
        return BGPU_OK;
    }
    const size_t nout = na + nb;
    if (nout > ((size_t)1 << 31)) return BGPU_ERR_CAPACITY;
    const size_t a_off = 0, b_off = align256(na * 8), o_off = b_off + align256(nb * 8);
    int rc = ensure(&g.d_io, &g.io_bytes, o_off + align256(nout * 8));
    if (rc != BGPU_OK) return rc;
    char* io = static_cast<char*>(g.d_io);
    uint64_t* da = reinterpret_cast<uint64_t*>(io + a_off);
    uint64_t* db = square ? da : reinterpret_cast<uint64_t*>(io + b_off);
    uint64_t* dout = reinterpret_cast<uint64_t*>(io + o_off);
    cudaStream_t st = g.stream;
    rc = host_to_device(da, a, na * 8, st, nullptr);
    if (rc == BGPU_OK && !square) rc = host_to_device(db, b, nb * 8, st, nullptr);
    if (rc != BGPU_OK) return rc;
    if (stats) cudaEventRecord(g.ev0, st);
    int fbits = 0, flog = 0;
    const bool want_fft = ((flags & BGPU_METHOD_MASK) == BGPU_METHOD_FFT || auto_fft(flags, na, nb)) &&
                          fft_pick(na, nb, flags, &fbits, &flog) == BGPU_OK;
    if (want_fft) {
        double err = 0;
        rc = fft_product_locked(da, na, db, nb, fbits, flog, dout, st, &err);
        if (rc != BGPU_OK) return rc;
        if (stats) {
            stats->method = BGPU_METHOD_FFT;
            stats->log2_points = (uint32_t)flog;
            stats->fft_bits = fbits;
            stats->max_round_err = err;
        }
        if (!(err <= kFftMaxErr)) {  // also catches NaN
            OperandDesc oa{da, (uint32_t)na, (uint32_t)(2 * na), kFmtLimb64};
            OperandDesc ob{db, (uint32_t)nb, (uint32_t)(2 * nb), kFmtLimb64};
            rc = multiply_device(oa, ob, square, dout, kFmtLimb64, nout, flags, st, nullptr);
            if (stats) stats->fell_back = 1;
        }
    } else if (const uint32_t sm = small_method(flags, na, nb)) {
        rc = launch_small(sm, da, na, db, nb, dout, st);
        g.last_launches = 1;
        if (stats) stats->method = (int32_t)sm;
    } else if (beyond_transform(na, nb)) {
        rc = huge_product(da, na, db, nb, dout, square, st);
        if (stats) stats->method = BGPU_METHOD_NTT;
    } else {
        OperandDesc oa{da, (uint32_t)na, (uint32_t)(2 * na), kFmtLimb64};
        OperandDesc ob{db, (uint32_t)nb, (uint32_t)(2 * nb), kFmtLimb64};
        rc = multiply_device(oa, ob, square, dout, kFmtLimb64, nout, flags, st, stats);
    }
    if (rc != BGPU_OK) return rc;
    if (stats) cudaEventRecord(g.ev1, st);
    // Copy straight into the caller's buffer when it holds na+nb limbs.
    std::vector<uint64_t> tmp;
    uint64_t* dst = out;
    if (out_cap < nout) {
        tmp.resize(nout);
        dst = tmp.data();
    }
    rc = device_to_host(dst, dout, nout * 8, st);
    rc = check_device_error(rc);
    if (rc != BGPU_OK) return rc;
    if (stats) cudaEventElapsedTime(&stats->device_ms, g.ev0, g.ev1);
    const size_t n = strip64(dst, nout);
    *out_len = n;
    if (dst != out) {
        if (n > out_cap) return BGPU_ERR_OUT_CAPACITY;
        memcpy(out, dst, n * 8);
    }
    return BGPU_OK;
}

// Product of device operands into dout (na + nb limbs, zero padded) with the
// method AUTO picks: a small-product kernel or the NTT.
int device_product(const uint64_t* da, size_t na, const uint64_t* db, size_t nb, uint64_t* dout,
                   cudaStream_t st, uint32_t* launches) {
    const bool square = da == db && na == nb;
    if (const uint32_t sm = small_method(BGPU_METHOD_AUTO, na, nb)) {
        *launches += 1;
        return launch_small(sm, da, na, db, nb, dout, st);
    }
    if (beyond_transform(na, nb)) return huge_product(da, na, db, nb, dout, square, st);
    OperandDesc oa{da, (uint32_t)na, (uint32_t)(2 * na), kFmtLimb64};
    OperandDesc ob{db, (uint32_t)nb, (uint32_t)(2 * nb), kFmtLimb64};
    *launches += kNttLaunches;
    return multiply_device(oa, ob, square, dout, kFmtLimb64, na + nb, BGPU_METHOD_AUTO, st, nullptr);
}

uint64_t bit_length(const uint64_t* x, size_t n) {  // n > 0, x[n-1] != 0
    return 64 * (uint64_t)(n - 1) + (64 - (uint64_t)__builtin_clzll(x[n - 1]));
}

// base^exponent by the reference's square-and-multiply (fast_pow<T>,
// include/bigint/bigint_base.h:60-69: res *= base on a set bit, then
// base *= base), every product on the device.  Operand lengths come from the
// exact bound bits(x y) <= bits(x) + bits(y), so the chain needs no host
// synchronisation; the final squaring the reference performs after the last
// set bit does not change the result and is skipped.
int pow_u64_locked(const uint64_t* base, size_t nbase, uint32_t exponent, uint64_t* out,
                   size_t out_cap, size_t* out_len) {
    nbase = strip64(base, nbase);
    if (exponent == 0 || (nbase == 1 && base[0] == 1)) {  // x^0 = 1 (the reference's res = 1)
        *out_len = 1;
        if (out_cap < 1) return BGPU_ERR_OUT_CAPACITY;
        out[0] = 1;
        return BGPU_OK;
    }
    if (nbase == 0) {
        *out_len = 0;
        return BGPU_OK;
    }
    const uint64_t bbits = bit_length(base, nbase);
    const uint64_t rbits = bbits * exponent;
    auto limbs = [](uint64_t bits) { return (size_t)((bits + 63) / 64); };
    const size_t rlimbs = limbs(rbits);
    if (rlimbs > ((size_t)1 << 30)) return BGPU_ERR_CAPACITY;
    // Plan the chain: operand sizes of every product, the largest transform.
    int max_ln = 0;
    size_t max_base = limbs(bbits);
    {
        uint64_t bb = bbits, rb = 0;
        for (uint32_t e = exponent; e; e >>= 1) {
            if (e & 1) {
                if (rb) {  // products beyond the largest transform run as its blocks
                    const uint64_t t32 = 2 * (uint64_t)(limbs(rb) + limbs(bb));
                    max_ln = std::max(max_ln, std::min(kMaxLogN, ceil_log2(t32 - 1)));
                }
                rb += bb;
            }
            if (e > 1) {
                const uint64_t t32 = 4 * (uint64_t)limbs(bb);
                max_ln = std::max(max_ln, std::min(kMaxLogN, ceil_log2(t32 - 1)));
                bb *= 2;
                max_base = std::max(max_base, limbs(bb));
            }
        }
    }
    // Device buffers: two for the running base, two for the running result.
    const size_t bsz = align256((2 * max_base + 2) * 8), rsz = align256((rlimbs + max_base + 2) * 8);
    int rc = ensure(&g.d_io, &g.io_bytes, 2 * bsz + 2 * rsz);
    if (rc != BGPU_OK) return rc;
    if (max_ln >= 5) {  // size the transform scratch once for the whole chain
        ProductScratch s{};
        rc = prepare_scratch(max_ln, false, &s);
        if (rc != BGPU_OK) return rc;
    }
    char* io = static_cast<char*>(g.d_io);
    uint64_t* bufb[2] = {reinterpret_cast<uint64_t*>(io), reinterpret_cast<uint64_t*>(io + bsz)};
    uint64_t* bufr[2] = {reinterpret_cast<uint64_t*>(io + 2 * bsz), reinterpret_cast<uint64_t*>(io + 2 * bsz + rsz)};
    cudaStream_t st = g.stream;
    rc = host_to_device(bufb[0], base, nbase * 8, st, nullptr);
    if (rc != BGPU_OK) return rc;
    cudaError_t e = cudaSuccess;
    int cb = 0, cr = 0;
    uint64_t bb = bbits, rb = 0;
    uint32_t nl = 0;
    for (uint32_t ex = exponent; ex; ex >>= 1) {
        if (ex & 1) {
            if (rb == 0) {
                e = cudaMemcpyAsync(bufr[cr], bufb[cb], limbs(bb) * 8, cudaMemcpyDeviceToDevice, st);
                if (e != cudaSuccess) return cuda_status(e);
            } else {
                rc = device_product(bufr[cr], limbs(rb), bufb[cb], limbs(bb), bufr[cr ^ 1], st, &nl);
                if (rc != BGPU_OK) return rc;
                cr ^= 1;
            }
            rb += bb;
        }
        if (ex > 1) {
            rc = device_product(bufb[cb], limbs(bb), bufb[cb], limbs(bb), bufb[cb ^ 1], st, &nl);
            if (rc != BGPU_OK) return rc;
            cb ^= 1;
            bb *= 2;
        }
    }
    g.last_launches = nl;
    std::vector<uint64_t> tmp;
    uint64_t* dst = out;
    if (out_cap < rlimbs) {
        tmp.resize(rlimbs);
        dst = tmp.data();
    }
    rc = device_to_host(dst, bufr[cr], rlimbs * 8, st);
    rc = check_device_error(rc);
    if (rc != BGPU_OK) return rc;
    const size_t n = strip64(dst, rlimbs);
    *out_len = n;
    if (dst != out) {
        if (n > out_cap) return BGPU_ERR_OUT_CAPACITY;
        memcpy(out, dst, n * 8);
    }
    return BGPU_OK;
}

// Many host-resident products, pipelined over four device slots (two for
// products above 256 MB): product i's operands go up on the H2D stream while
// earlier products compute and their results come back on the D2H stream.
// Every product still makes its own host->device and device->host copies.
int mul_u64_many_locked(const bgpu_host_product* p, size_t count, uint32_t flags) {
    struct Item { size_t na, nb; bool square; };
    std::vector<Item> it(count);
    size_t slot_in = 0, slot_out = 0;
    int max_ln = 0;
    for (size_t i = 0; i < count; ++i) {
        const bgpu_host_product& q = p[i];
        if (!q.a || !q.b || !q.out || !q.out_len || q.na == 0 || q.nb == 0) return BGPU_ERR_INVALID_ARG;
        const bool square = q.a == q.b && q.na == q.nb;
        const size_t na = strip64(q.a, q.na), nb = square ? na : strip64(q.b, q.nb);
        if (q.out_cap < q.na + q.nb) return BGPU_ERR_OUT_CAPACITY;
        if (na + nb > ((size_t)1 << 31)) return BGPU_ERR_CAPACITY;
        it[i] = {na, nb, square};
        slot_in = std::max(slot_in, align256(na * 8) + align256(nb * 8));
        slot_out = std::max(slot_out, align256((na + nb) * 8));
        if (na && nb && !small_method(flags, na, nb)) {  // beyond the largest transform: its blocks
            const int ln = std::min(kMaxLogN, ceil_log2(2 * (uint64_t)(na + nb) - 1));
            max_ln = std::max(max_ln, ln < 5 ? 5 : ln);
        }
    }
    const size_t slot = slot_in + slot_out;
    // Four device slots keep both copy directions busy (the upload of
    // product i waits only for the download of product i - 4); products
    // above 256 MB of operands and result use two.
    const size_t nslots = slot <= ((size_t)256 << 20) ? 4 : 2;
    int rc = ensure(&g.d_many, &g.many_bytes, nslots * slot);
    if (rc != BGPU_OK) return rc;
    if (max_ln) {  // size the transform scratch once, before anything is in flight
        ProductScratch s{};
        rc = prepare_scratch(max_ln, false, &s);
        if (rc != BGPU_OK) return rc;
    }
    cudaStream_t st = g.stream;
    uint32_t nl = 0;
    for (size_t i = 0; i < count; ++i) {
        const bgpu_host_product& q = p[i];
        const Item& m = it[i];
        const int k = (int)(i % nslots);
        char* base = static_cast<char*>(g.d_many) + k * slot;
        uint64_t* da = reinterpret_cast<uint64_t*>(base);
        uint64_t* db = m.square ? da : reinterpret_cast<uint64_t*>(base + align256(m.na * 8));
        uint64_t* dout = reinterpret_cast<uint64_t*>(base + slot_in);
        const size_t nout = q.na + q.nb;
        cudaError_t e = cudaSuccess;
        if (i >= nslots) e = cudaStreamWaitEvent(g.h2d, g.ev_out[k], 0);  // slot k's last result is out
        if (m.na == 0 || m.nb == 0) {  // a zero operand: the product is zero
            if (e == cudaSuccess) e = cudaMemsetAsync(dout, 0, nout * 8, g.h2d);
            if (e == cudaSuccess) e = cudaEventRecord(g.ev_comp[k], g.h2d);
        } else {
            if (e == cudaSuccess) e = cudaMemcpyAsync(da, q.a, m.na * 8, cudaMemcpyHostToDevice, g.h2d);
            if (e == cudaSuccess && !m.square)
                e = cudaMemcpyAsync(db, q.b, m.nb * 8, cudaMemcpyHostToDevice, g.h2d);
            if (e == cudaSuccess) e = cudaEventRecord(g.ev_in[k], g.h2d);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(st, g.ev_in[k], 0);
            if (e != cudaSuccess) return cuda_status(e);
            if (const uint32_t sm = small_method(flags, m.na, m.nb)) {
                rc = launch_small(sm, da, m.na, db, m.nb, dout, st);
                nl += 1;
            } else if (beyond_transform(m.na, m.nb)) {
                rc = huge_product(da, m.na, db, m.nb, dout, m.square, st);
            } else {
                OperandDesc oa{da, (uint32_t)m.na, (uint32_t)(2 * m.na), kFmtLimb64};
                OperandDesc ob{db, (uint32_t)m.nb, (uint32_t)(2 * m.nb), kFmtLimb64};
                rc = multiply_device(oa, ob, m.square, dout, kFmtLimb64, m.na + m.nb, flags, st, nullptr);
                nl += kNttLaunches;
            }
            if (rc != BGPU_OK) return rc;
            if (m.na + m.nb < nout) e = cudaMemsetAsync(dout + m.na + m.nb, 0, (nout - m.na - m.nb) * 8, st);
            if (e == cudaSuccess) e = cudaEventRecord(g.ev_comp[k], st);
        }
        if (e == cudaSuccess) e = cudaStreamWaitEvent(g.d2h, g.ev_comp[k], 0);
        // The product goes back in pieces the size of the larger operand's
        // upload.  With copies of equal size in flight both ways the copy
        // engines share the link evenly; one 4 MiB download against 2 MiB
        // uploads left the uploads at 31 GB/s (measured at 2^24-bit
        // products: 137 us per product, 122 us with two 2 MiB pieces;
        // smaller pieces were slower again).
        const size_t piece = std::max<size_t>(std::max(m.na, m.nb), 4096) * 8;
        for (size_t off = 0; e == cudaSuccess && off < nout * 8; off += piece)
            e = cudaMemcpyAsync(reinterpret_cast<char*>(q.out) + off, reinterpret_cast<const char*>(dout) + off,
                                std::min(piece, nout * 8 - off), cudaMemcpyDeviceToHost, g.d2h);
        if (e == cudaSuccess) e = cudaEventRecord(g.ev_out[k], g.d2h);
        if (e != cudaSuccess) return cuda_status(e);
    }
    g.last_launches = nl;
    cudaError_t e = cudaStreamSynchronize(g.d2h);
    if (e != cudaSuccess) return cuda_status(e);
    rc = check_device_error(BGPU_OK);
    if (rc != BGPU_OK) return rc;
    for (size_t i = 0; i < count; ++i) *p[i].out_len = strip64(p[i].out, p[i].na + p[i].nb);
    return BGPU_OK;
}

int mul_digits_locked(const uint32_t* a, size_t na, const uint32_t* b, size_t nb, size_t prec,
                      int64_t* point_pos, uint32_t* out, size_t out_cap, size_t* out_len,
                      uint32_t flags, bgpu_stats* stats) {
    const bool square = (a == b && na == nb);
    if (stats) memset(stats, 0, sizeof(*stats));
    // Offsets exactly as mul_digits (include/bigint/mul.h:227-243).
    size_t off_a = (prec == 0 || na <= prec) ? 0 : na - prec;
    size_t off_b = (prec == 0 || nb <= prec) ? 0 : nb - prec;
    size_t tz_a = 0, tz_b = 0;
    while (off_a + tz_a < na && a[off_a + tz_a] == 0) ++tz_a;
    if (off_a + tz_a == na) return BGPU_ERR_INVALID_ARG;
    if (square) {
        tz_b = tz_a;
    } else {
        while (off_b + tz_b < nb && b[off_b + tz_b] == 0) ++tz_b;
        if (off_b + tz_b == nb) return BGPU_ERR_INVALID_ARG;
    }
    off_a += tz_a;
    off_b += tz_b;
    const uint32_t* pa = a + off_a;
    const uint32_t* pb = b + off_b;
    size_t la = strip32(pa, na - off_a), lb = square ? la : strip32(pb, nb - off_b);
    const size_t nres = la + lb + 1;  // 28-bit digits of the product, with margin
    if (nres > ((size_t)1 << 31)) return BGPU_ERR_CAPACITY;
    const size_t la64 = (la * 28 + 63) / 64, lb64 = (lb * 28 + 63) / 64;
    const size_t a_off = 0, b_off = align256(la * 4), o_off = b_off + align256(lb * 4);
    const size_t l_off = o_off + align256(nres * 4);
    const size_t need = l_off + align256((la64 + 1) * 8) + align256((lb64 + 1) * 8) +
                        align256((la64 + lb64) * 8);
    int rc = ensure(&g.d_io, &g.io_bytes, need);
    if (rc != BGPU_OK) return rc;
    char* io = static_cast<char*>(g.d_io);
    uint32_t* da = reinterpret_cast<uint32_t*>(io + a_off);
    uint32_t* db = square ? da : reinterpret_cast<uint32_t*>(io + b_off);
    uint32_t* dres = reinterpret_cast<uint32_t*>(io + o_off);
    cudaStream_t st = g.stream;
    // the 28-bit check rides on the copies; nothing is launched before it
    bool ok_a = true, ok_b = true;
    rc = host_to_device(da, pa, la * 4, st, &ok_a);
    if (rc == BGPU_OK && !square) rc = host_to_device(db, pb, lb * 4, st, &ok_b);
    if (rc != BGPU_OK) return rc;
    if (!ok_a || !ok_b) {
        cudaStreamSynchronize(st);  // a page-locked source may still be in flight
        return BGPU_ERR_INVALID_ARG;
    }
    cudaError_t e = cudaSuccess;
    if (stats) cudaEventRecord(g.ev0, st);
    // Small products run on u64 limbs; so do products beyond the largest
    // transform (blocks of NTT products, huge.cu).
    const uint32_t sm = small_method(flags, la64, lb64);
    const uint64_t n32 = (bits28(pa, la) + 31) / 32 + (bits28(pb, lb) + 31) / 32;
    const bool huge = !sm && ceil_log2(n32 - 1) > transform_cap_log();
    if (sm || huge) {
        uint64_t* la_d = reinterpret_cast<uint64_t*>(io + l_off);
        uint64_t* lb_d = square ? la_d : la_d + align256((la64 + 1) * 8) / 8;
        uint64_t* lo_d = reinterpret_cast<uint64_t*>(io + l_off + align256((la64 + 1) * 8) +
                                                     align256((lb64 + 1) * 8));
        e = launch_digits28_to_limbs(da, (uint32_t)la, la_d, (uint32_t)la64, st);
        if (e == cudaSuccess && !square)
            e = launch_digits28_to_limbs(db, (uint32_t)lb, lb_d, (uint32_t)lb64, st);
        rc = cuda_status(e);
        if (rc == BGPU_OK)
            rc = sm ? launch_small(sm, la_d, la64, lb_d, lb64, lo_d, st)
                    : huge_product(la_d, la64, lb_d, lb64, lo_d, square, st);
        if (rc == BGPU_OK)
            rc = cuda_status(launch_limbs_to_digits28(lo_d, (uint32_t)(la64 + lb64), dres, (uint32_t)nres, st));
        g.last_launches = square ? 3 : 4;
        if (stats) stats->method = sm ? (int32_t)sm : BGPU_METHOD_NTT;
    } else {
        // 32-bit digit counts from the true bit lengths: a number of exactly
        // 2^k bits has ceil(2^k / 28) digits, whose 28 * digits overshoots 2^k
        // and would double the transform
        OperandDesc oa{da, (uint32_t)la, (uint32_t)((bits28(pa, la) + 31) / 32), kFmtDigit28};
        OperandDesc ob{db, (uint32_t)lb, (uint32_t)((bits28(pb, lb) + 31) / 32), kFmtDigit28};
        rc = multiply_device(oa, ob, square, dres, kFmtDigit28, nres, flags, st, stats);
    }
    if (rc != BGPU_OK) return rc;
    if (stats) cudaEventRecord(g.ev1, st);
    // Result digits land in the caller's buffer when it is large enough.
    const size_t z = prec ? 0 : tz_a + tz_b;
    std::vector<uint32_t> tmp;
    uint32_t* dst = (out_cap >= z + nres) ? out + z : nullptr;
    if (!dst) {
        tmp.resize(nres);
        dst = tmp.data();
    }
    rc = device_to_host(dst, dres, nres * 4, st);
    rc = check_device_error(rc);
    if (rc != BGPU_OK) return rc;
    if (stats) cudaEventElapsedTime(&stats->device_ms, g.ev0, g.ev1);
    size_t n = strip32(dst, nres);
    if (prec) {
        // Trim to the top digits and shift the point (include/bigint/mul.h:302-312).
        size_t off_r = n <= prec ? 0 : n - prec;
        while (dst[off_r] == 0) ++off_r;
        const size_t keep = n - off_r;
        if (point_pos) *point_pos -= (int64_t)(off_a + off_b + off_r);
        *out_len = keep;
        if (keep > out_cap) return BGPU_ERR_OUT_CAPACITY;
        memmove(out, dst + off_r, keep * 4);
    } else {
        *out_len = z + n;
        if (z + n > out_cap) return BGPU_ERR_OUT_CAPACITY;
        if (dst != out + z) memcpy(out + z, dst, n * 4);
        memset(out, 0, z * 4);
    }
    return BGPU_OK;
}


// ---- device-resident BigFloat::reciprocal ----------------------------------
//
// The reference's Newton iteration (src/bigint.cpp:1044-1071):
//   b = *this >> exponent, tail zeros removed (b in [1/2, 1));
//   x = BigFloat(1 / b.to_double());
//   while (cur < precision) { cur *= 2;
//       x += mul(x, one - mul(b, x, cur + 1), cur + 1); }
//   return x >> exponent;
// replayed step by step with every value's digits on the device.  The host
// keeps what the reference's control flow reads -- each value's length, point
// position, sign, bottom zeros and top digit -- and gets it back after each
// step from the extent kernel (four words); the digit work runs in device
// kernels: truncated products (BigFloat::mul -> mul_digits) on the NTT or the
// small-product kernels, frame additions and subtractions (add_or_sub) and
// shifts.  Only the starting value 1 / b.to_double() (two or three digits)
// is formed on the host, from b's top three digits, as the reference does.

enum RecipSlot {
    kRsIn, kRsB, kRsX0, kRsX1, kRsT1, kRsT2, kRsT3, kRsOut, kRsScratch, kRsSmall, kRsOne,
    // divmod: the operands, the quotient estimate, Q, Q * b, R and the adjusted Q and R
    kRsDivA, kRsDivB, kRsDivP, kRsDivQ, kRsDivQB, kRsDivR, kRsDivQ2, kRsDivR2,
    // small powers (BigFloat::print's 5^d): running base and result, two each
    kRsPowB0, kRsPowB1, kRsPowR0, kRsPowR1, kRsSlots
};

constexpr uint32_t kDigitMask = (1u << 28) - 1u;

struct DVal {
    const uint32_t* d = nullptr;  // d[0..n); the zero value is {0} and has no digits on the device
    size_t n = 1;
    int64_t pp = 0;               // point position: value = digits * 2^(-28 pp)
    bool neg = false;
    size_t tz = 0;                // zero digits at the bottom
    uint32_t top = 0;             // d[n-1]
    int slot = -1;                // buffer holding the digits (-1: none)
    bool zero() const { return n == 1 && top == 0; }
};

static_assert(kRsSlots == sizeof(Engine::rs) / sizeof(Engine::rs[0]), "one buffer per slot");

uint32_t* rslot(int k, size_t words, int* rc) {
    *rc = ensure(reinterpret_cast<void**>(&g.rs[k]), &g.rs_bytes[k], std::max<size_t>(words, 4) * 4);
    return *rc == BGPU_OK ? g.rs[k] : nullptr;
}

// Runs what is queued and reads `count` words back.
// Small readbacks go through one page-locked block (a pageable copy costs a
// driver staging pass per call).  Device errors are not read here: the
// callers check the sticky error word once, at the end or on failure.
unsigned long long* small_host() {
    if (!g.h_small && cudaHostAlloc(reinterpret_cast<void**>(&g.h_small), 64, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        g.h_small = nullptr;
    }
    return g.h_small;
}

int read_back(const uint32_t* d, uint32_t* h, size_t count) {
    unsigned long long* hp = count <= 16 ? small_host() : nullptr;
    void* dst = hp ? static_cast<void*>(hp) : static_cast<void*>(h);
    cudaError_t e = cudaMemcpyAsync(dst, d, count * 4, cudaMemcpyDeviceToHost, g.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g.stream);
    if (e == cudaSuccess && hp) memcpy(h, hp, count * 4);
    return cuda_status(e);
}

// The four-word result block of the compare and extent kernels, zeroed.
int result_block(unsigned long long** dr) {
    int rc;
    uint32_t* p = rslot(kRsSmall, 8, &rc);
    if (rc != BGPU_OK) return rc;
    *dr = reinterpret_cast<unsigned long long*>(p);
    return cuda_status(cudaMemsetAsync(p, 0, 4 * sizeof(unsigned long long), g.stream));
}

// Queues the extent kernel into the block, runs everything queued and reads
// the block back: r[0] = highest nonzero index + 1 (0: all zero), r[1], r[2] =
// lowest nonzero index >= from0, from1 (0xffffffff: none), r[3] = the digit
// at r[0] - 1; *cmp (if given) = the compare word.
int extent(unsigned long long* dr, const uint32_t* d, size_t n, size_t from0, size_t from1, uint32_t r[4],
           unsigned long long* cmp = nullptr) {
    cudaError_t e = launch_extent(d, (uint32_t)n, (uint32_t)std::min<size_t>(from0, UINT32_MAX),
                                  (uint32_t)std::min<size_t>(from1, UINT32_MAX), dr, g.stream);
    if (e != cudaSuccess) return cuda_status(e);
    unsigned long long h[4];
    const int rc = read_back(reinterpret_cast<const uint32_t*>(dr), reinterpret_cast<uint32_t*>(h), 8);
    if (rc != BGPU_OK) return rc;
    r[0] = (uint32_t)(h[0] >> 32);
    r[3] = (uint32_t)h[0];
    r[1] = h[1] ? (uint32_t)((1ull << 32) - h[1]) : 0xffffffffu;
    r[2] = h[2] ? (uint32_t)((1ull << 32) - h[2]) : 0xffffffffu;
    if (cmp) *cmp = h[3];
    return BGPU_OK;
}

// BigFloat::shift (src/bigint.cpp:769-789): the point moves by whole digits
// (C++ division, truncating toward zero), the remaining bits by a right shift
// when the bottom digit has that many zero bits, else by a left shift.
struct ShiftPlan {
    int64_t pp;
    int mode;  // 0 none, 1 right by s, 2 left by s
    uint32_t s;
};

ShiftPlan plan_shift(int64_t pp, int64_t offset, uint32_t low) {
    pp -= offset / 28;
    int64_t off = offset % 28;
    if (off == 0) return {pp, 0, 0};
    if (off > 0) {
        off = 28 - off;
        --pp;
    } else {
        off = -off;
    }
    const int64_t ctz = low ? __builtin_ctz(low) : 32;
    if (ctz >= off) return {pp, 1, (uint32_t)off};
    return {pp + 1, 2, (uint32_t)(28 - off)};
}

// The same on a short host vector (the double-derived starting value).
void host_shift(std::vector<uint32_t>& v, int64_t* pp, bool* neg, int64_t offset) {
    const ShiftPlan sp = plan_shift(*pp, offset, v[0]);
    *pp = sp.pp;
    const size_t n = v.size();
    if (sp.mode == 1) {
        for (size_t i = 0; i + 1 < n; ++i) v[i] = ((v[i] >> sp.s) | (v[i + 1] << (28 - sp.s))) & kDigitMask;
        v[n - 1] >>= sp.s;
    } else if (sp.mode == 2) {
        v.push_back(0);
        for (size_t i = n; i > 0; --i) v[i] = ((v[i] << sp.s) | (v[i - 1] >> (28 - sp.s))) & kDigitMask;
        v[0] = (v[0] << sp.s) & kDigitMask;
    }
    size_t i = v.size();
    while (i > 1 && v[i - 1] == 0) --i;
    v.resize(i);
    if (i == 1 && v[0] == 0) {  // reset()
        *pp = 0;
        *neg = false;
    }
}

// BigFloat::to_double (src/bigint.cpp:717-766) from the top k <= 3 digits
// t[0..k) of an n-digit value (t[k-1] = top); b in [1/2, 1) needs at most two
// digits below the top.
double to_double_top(const uint32_t* t, size_t k, size_t n, int64_t pp, bool neg, bool* ok) {
    auto dig = [&](size_t i) { return (uint64_t)t[i - (n - k)]; };
    auto shl = [](uint64_t x, int64_t r) { return r < 0 ? x >> (-r) : x << r; };
    const uint32_t top = t[k - 1];
    const int64_t hbw = 32 - __builtin_clz(top);
    const int64_t exponent = 28 * ((int64_t)n - 1 - pp) + hbw - 1;
    int64_t eb = exponent + 1023;
    *ok = true;
    if (eb >= 2047) return neg ? -HUGE_VAL : HUGE_VAL;
    int64_t offset;
    uint64_t mant;
    if (eb <= 0) {
        if (exponent < -52 - 1023 + 1) return neg ? -0.0 : 0.0;
        eb = 0;
        offset = exponent + 52 + 1023 - hbw;
        mant = shl(top, offset);
    } else {
        offset = 52 - (hbw - 1);
        mant = shl(top & ((1u << (hbw - 1)) - 1), offset);
    }
    size_t i = n - 1;
    while (offset > 0 && i > 0) {
        offset -= 28;
        --i;
        if (i < n - k) {  // needs more than the top three digits
            *ok = false;
            return 0.0;
        }
        mant |= shl(dig(i), offset);
    }
    const uint64_t bits = ((uint64_t)neg << 63) | ((uint64_t)eb << 52) | mant;
    double r;
    memcpy(&r, &bits, sizeof(r));
    return r;
}

// BigFloat::BigFloat(double) (src/bigint.cpp:681-715) for finite nonzero v.
void double_to_digits(double v, std::vector<uint32_t>* d, int64_t* pp, bool* neg) {
    uint64_t raw;
    memcpy(&raw, &v, sizeof(raw));
    *pp = 0;
    *neg = (raw >> 63) != 0;
    const int64_t eb = (int64_t)((raw >> 52) & 2047);
    uint64_t base = raw & ((1ull << 52) - 1);
    int64_t offset = -52 - 1023;
    if (eb == 0) {
        offset += 1;
    } else {
        base |= 1ull << 52;
        offset += eb;
    }
    d->clear();
    while (base) {
        d->push_back((uint32_t)base & kDigitMask);
        base >>= 28;
    }
    host_shift(*d, pp, neg, offset);
}

// *out = in shifted as BigFloat::shift(offset) does, into `slot`.
int shift_val(const DVal& in, int64_t offset, int slot, DVal* out) {
    uint32_t low = 0;
    int rc = read_back(in.d, &low, 1);
    if (rc != BGPU_OK) return rc;
    const ShiftPlan sp = plan_shift(in.pp, offset, low);
    *out = in;
    out->pp = sp.pp;
    if (sp.mode == 0) return BGPU_OK;  // whole digits: only the point moves
    const size_t nout = in.n + (sp.mode == 2 ? 1 : 0);
    uint32_t* o = rslot(slot, nout, &rc);
    if (rc != BGPU_OK) return rc;
    unsigned long long* dr = nullptr;
    rc = cuda_status(launch_shift_digits(in.d, (uint32_t)in.n, sp.s, sp.mode == 2, o, g.stream));
    if (rc == BGPU_OK) rc = result_block(&dr);
    uint32_t r[4];
    if (rc == BGPU_OK) rc = extent(dr, o, nout, 0, 0, r);
    if (rc != BGPU_OK) return rc;
    if (r[0] == 0) return BGPU_ERR_CUDA;  // a nonzero value cannot shift to zero
    out->d = o;
    out->n = r[0];
    out->tz = r[1];
    out->top = r[3];
    out->slot = slot;
    return BGPU_OK;
}

// Product of the device digit ranges a.d[off_a..a.n) and b.d[off_b..b.n)
// into nres digits at dres, by the method the host API would use.
int digits_product(const DVal& a, size_t off_a, const DVal& b, size_t off_b, uint32_t* dres, size_t nres) {
    const uint32_t* pa = a.d + off_a;
    const uint32_t* pb = b.d + off_b;
    const size_t la = a.n - off_a, lb = b.n - off_b;
    const size_t la64 = (la * 28 + 63) / 64, lb64 = (lb * 28 + 63) / 64;
    cudaStream_t st = g.stream;
    const uint64_t bits_a = 28 * (uint64_t)(la - 1) + (32 - __builtin_clz(a.top));
    const uint64_t bits_b = 28 * (uint64_t)(lb - 1) + (32 - __builtin_clz(b.top));
    const uint32_t sm = small_method(BGPU_METHOD_AUTO, la64, lb64);
    const bool huge = !sm && ceil_log2((bits_a + 31) / 32 + (bits_b + 31) / 32 - 1) > transform_cap_log();
    if (sm || huge) {  // on u64 limbs: the small kernels, or NTT blocks beyond the largest transform
        int rc;
        uint32_t* scr = rslot(kRsScratch, 2 * ((la64 + 1) + (lb64 + 1) + (la64 + lb64)), &rc);
        if (rc != BGPU_OK) return rc;
        uint64_t* la_d = reinterpret_cast<uint64_t*>(scr);
        uint64_t* lb_d = la_d + la64 + 1;
        uint64_t* lo_d = lb_d + lb64 + 1;
        cudaError_t e = launch_digits28_to_limbs(pa, (uint32_t)la, la_d, (uint32_t)la64, st);
        if (e == cudaSuccess) e = launch_digits28_to_limbs(pb, (uint32_t)lb, lb_d, (uint32_t)lb64, st);
        rc = cuda_status(e);
        if (rc == BGPU_OK)
            rc = sm ? launch_small(sm, la_d, la64, lb_d, lb64, lo_d, st)
                    : huge_product(la_d, la64, lb_d, lb64, lo_d, false, st);
        if (rc == BGPU_OK)
            rc = cuda_status(launch_limbs_to_digits28(lo_d, (uint32_t)(la64 + lb64), dres, (uint32_t)nres, st));
        return rc;
    }
    OperandDesc oa{pa, (uint32_t)la, (uint32_t)((bits_a + 31) / 32), kFmtDigit28};
    OperandDesc ob{pb, (uint32_t)lb, (uint32_t)((bits_b + 31) / 32), kFmtDigit28};
    return multiply_device(oa, ob, false, dres, kFmtDigit28, nres, BGPU_METHOD_AUTO, st, nullptr);
}

// BigFloat::mul(a, b, prec) (include/bigint/bigint.h:570-582) with the
// truncation of mul_digits (include/bigint/mul.h:227-243, 301-312).  The
// truncated operands keep any zero digits at their bottom: the product then
// carries those zeros below its own digits, and the first nonzero digit at or
// above the cut lands where the reference's cut and zero skip put it.
int mul_trunc(const DVal& a, const DVal& b, size_t prec, int slot, DVal* out) {
    if (a.zero() || b.zero()) {
        *out = DVal{};
        return BGPU_OK;
    }
    const size_t off_a = a.n > prec ? a.n - prec : 0, off_b = b.n > prec ? b.n - prec : 0;
    const size_t la = a.n - off_a, lb = b.n - off_b;
    const size_t nres = la + lb + 1;
    if (nres > ((size_t)1 << 31)) return BGPU_ERR_CAPACITY;
    int rc;
    uint32_t* dres = rslot(slot, nres, &rc);
    if (rc != BGPU_OK) return rc;
    unsigned long long* dr = nullptr;
    rc = digits_product(a, off_a, b, off_b, dres, nres);
    if (rc == BGPU_OK) rc = result_block(&dr);
    if (rc != BGPU_OK) return rc;
    // the product has la + lb - 1 or la + lb digits
    const size_t n0 = la + lb - 1, n1 = la + lb;
    uint32_t r[4];
    rc = extent(dr, dres, nres, n0 > prec ? n0 - prec : 0, n1 > prec ? n1 - prec : 0, r);
    if (rc != BGPU_OK) return rc;
    const uint32_t first = r[0] == n0 ? r[1] : (r[0] == n1 ? r[2] : 0xffffffffu);
    if (first >= r[0]) return BGPU_ERR_CUDA;
    out->d = dres + first;
    out->n = r[0] - first;
    out->pp = a.pp + b.pp - (int64_t)(off_a + off_b + first);
    out->neg = a.neg != b.neg;
    out->tz = 0;
    out->top = r[3];
    out->slot = slot;
    return BGPU_OK;
}

// BigFloat::add_or_sub (src/bigint.cpp:849-936): the exact sum or difference
// in the reference's frame, then its leading and bottom zeros removed.
int add_or_sub(const DVal& a, const DVal& b, bool is_sub, int slot, DVal* out) {
    if (a.zero()) {
        *out = b;
        if (is_sub && !b.zero()) out->neg = !b.neg;
        return BGPU_OK;
    }
    if (b.zero()) {
        *out = a;
        return BGPU_OK;
    }
    const int64_t len_a = (int64_t)a.n, len_b = (int64_t)b.n;
    const int64_t pp_res = std::max(a.pp - (int64_t)a.tz, b.pp - (int64_t)b.tz);
    const int64_t len_res = std::max(len_a - a.pp, len_b - b.pp) + pp_res;
    if (len_res <= 0 || len_res >= ((int64_t)1 << 31)) return BGPU_ERR_CAPACITY;
    FrameOp f{a.d, pp_res - a.pp, (uint32_t)a.n, b.d, pp_res - b.pp, (uint32_t)b.n, (uint32_t)len_res, 0,
              nullptr};
    const bool sub = a.neg != (b.neg != is_sub);  // magnitudes subtract
    const uint32_t L = (uint32_t)len_res, nblk = frame_blocks(L);
    const size_t dig = (L + 1 + 63) & ~(size_t)63;
    int rc;
    uint32_t* o = rslot(slot, dig + 2 * (size_t)nblk, &rc);
    unsigned long long* dr = nullptr;
    if (rc == BGPU_OK) rc = result_block(&dr);
    if (rc != BGPU_OK) return rc;
    if (sub) {
        // the compare stays on the device: the frame kernels read it and
        // subtract the smaller magnitude from the larger (the reference's
        // negation when B is larger); equal magnitudes give all-zero digits
        rc = cuda_status(launch_frame_cmp(f, dr + 3, g.stream));
        f.sub = 1;
        f.order = dr + 3;
    }
    if (rc == BGPU_OK) rc = cuda_status(launch_frame_addsub(f, o + dig, o + dig + nblk, o, g.stream));
    uint32_t r[4];
    unsigned long long cmp = 0;
    if (rc == BGPU_OK) rc = extent(dr, o, L + 1, 0, 0, r, &cmp);
    if (rc != BGPU_OK) return rc;
    if (sub && cmp == 0) {  // exactly zero: reset()
        *out = DVal{};
        return BGPU_OK;
    }
    if (r[0] == 0 || r[1] >= r[0]) return BGPU_ERR_CUDA;  // a nonzero result has a nonzero digit
    out->d = o + r[1];
    out->n = r[0] - r[1];
    out->pp = pp_res - (int64_t)r[1];
    out->neg = sub && (cmp & 3u) == 2u ? !a.neg : a.neg;
    out->tz = 0;
    out->top = r[3];
    out->slot = slot;
    return BGPU_OK;
}

int upload_digits(int slot, const std::vector<uint32_t>& v, int64_t pp, bool neg, DVal* out) {
    int rc;
    uint32_t* d = rslot(slot, v.size(), &rc);
    if (rc != BGPU_OK) return rc;
    rc = cuda_status(cudaMemcpyAsync(d, v.data(), v.size() * 4, cudaMemcpyHostToDevice, g.stream));
    if (rc == BGPU_OK) rc = cuda_status(cudaStreamSynchronize(g.stream));
    if (rc != BGPU_OK) return rc;
    size_t tz = 0;
    while (tz < v.size() && v[tz] == 0) ++tz;
    *out = DVal{d, v.size(), pp, neg, tz, v.back(), slot};
    return BGPU_OK;
}

int reciprocal_steps(const uint32_t* digits, size_t n, int64_t point_pos, bool neg, size_t precision,
                     uint32_t* out, size_t out_cap, size_t* out_len, int64_t* out_pp, int* out_neg);
int reciprocal_val(const DVal& in, size_t precision, DVal* res);

// A failed step-by-step call reports a device-side error (sticky, e.g. a
// carry-scan timeout in one of its products) in preference to what the
// failure looked like on the host, and leaves the error word clear.
int with_device_status(int rc) {
    if (rc == BGPU_OK || rc == BGPU_ERR_OUT_CAPACITY) return rc;
    cudaStreamSynchronize(g.stream);
    const int dev = check_device_error(BGPU_OK);
    return dev != BGPU_OK ? dev : rc;
}

int reciprocal_locked(const uint32_t* digits, size_t n, int64_t point_pos, bool neg, size_t precision,
                      uint32_t* out, size_t out_cap, size_t* out_len, int64_t* out_pp, int* out_neg) {
    return with_device_status(reciprocal_steps(digits, n, point_pos, neg, precision, out, out_cap, out_len,
                                               out_pp, out_neg));
}

int reciprocal_steps(const uint32_t* digits, size_t n, int64_t point_pos, bool neg, size_t precision,
                     uint32_t* out, size_t out_cap, size_t* out_len, int64_t* out_pp, int* out_neg) {
    if (n >= ((size_t)1 << 31)) return BGPU_ERR_CAPACITY;
    for (size_t i = 0; i < n; ++i)
        if (digits[i] >> 28) return BGPU_ERR_INVALID_ARG;
    if (digits[n - 1] == 0) return BGPU_ERR_INVALID_ARG;  // a leading zero digit, or the value zero
    if (precision == 0) precision = n;
    int rc;
    uint32_t* din = rslot(kRsIn, n, &rc);
    if (rc != BGPU_OK) return rc;
    rc = host_to_device(din, digits, n * 4, g.stream, nullptr);
    if (rc != BGPU_OK) return rc;
    size_t tz = 0;
    while (digits[tz] == 0) ++tz;
    const DVal in{din, n, point_pos, neg, tz, digits[n - 1], kRsIn};
    DVal r;
    rc = reciprocal_val(in, precision, &r);
    if (rc != BGPU_OK) return rc;
    *out_len = r.n;
    *out_pp = r.pp;
    *out_neg = r.neg ? 1 : 0;
    if (r.n > out_cap) return BGPU_ERR_OUT_CAPACITY;
    rc = device_to_host(out, r.d, r.n * 4, g.stream);
    return check_device_error(rc);
}

// in.reciprocal(precision) with the value's digits on the device; the result
// lies in one of the reciprocal's own slots (kRsX0, kRsX1 or kRsOut).
int reciprocal_val(const DVal& in, size_t precision, DVal* res) {
    const int64_t exponent = 28 * ((int64_t)in.n - 1 - in.pp) + (32 - __builtin_clz(in.top));
    int rc;

    // b = *this >> exponent; b.remove_tail_zero()
    DVal b;
    rc = shift_val(in, -exponent, kRsB, &b);
    if (rc != BGPU_OK) return rc;
    b.d += b.tz;
    b.n -= b.tz;
    b.pp -= (int64_t)b.tz;
    b.tz = 0;

    // x = BigFloat(1 / b.to_double())
    uint32_t t[3];
    const size_t k = std::min<size_t>(b.n, 3);
    rc = read_back(b.d + (b.n - k), t, k);
    if (rc != BGPU_OK) return rc;
    bool ok;
    const double bd = to_double_top(t, k, b.n, b.pp, b.neg, &ok);
    if (!ok || !(std::fabs(bd) >= 0.5 && std::fabs(bd) < 1.0)) return BGPU_ERR_CUDA;
    std::vector<uint32_t> x0;
    int64_t x0_pp;
    bool x0_neg;
    double_to_digits(1 / bd, &x0, &x0_pp, &x0_neg);
    DVal x, one;
    rc = upload_digits(kRsX0, x0, x0_pp, x0_neg, &x);
    if (rc == BGPU_OK) rc = upload_digits(kRsOne, std::vector<uint32_t>{1u}, 0, false, &one);
    if (rc != BGPU_OK) return rc;

    size_t cur = 52 / 28;  // DOUBLE_MANTISSA_LEN / DIGIT_BITS
    while (cur < precision) {
        cur *= 2;
        DVal t1, t2, t3, xn;
        rc = mul_trunc(b, x, cur + 1, kRsT1, &t1);
        if (rc == BGPU_OK) rc = add_or_sub(one, t1, true, kRsT2, &t2);
        if (rc == BGPU_OK) rc = mul_trunc(x, t2, cur + 1, kRsT3, &t3);
        const int xs = x.slot == kRsX0 ? kRsX1 : kRsX0;
        if (rc == BGPU_OK) rc = add_or_sub(x, t3, false, xs, &xn);
        if (rc != BGPU_OK) return rc;
        if (xn.slot != kRsX0 && xn.slot != kRsX1) {  // x + t3 returned t3 itself: keep x in an x buffer
            uint32_t* d = rslot(xs, xn.n, &rc);
            if (rc != BGPU_OK) return rc;
            if (!xn.zero()) {
                rc = cuda_status(cudaMemcpyAsync(d, xn.d, xn.n * 4, cudaMemcpyDeviceToDevice, g.stream));
                if (rc != BGPU_OK) return rc;
                xn.d = d;
            }
            xn.slot = xs;
        }
        x = xn;
    }

    // x >>= exponent
    if (x.zero()) return BGPU_ERR_CUDA;
    return shift_val(x, -exponent, kRsOut, res);
}

// ---- BigInt::divmod (src/bigint.cpp:625-673) ----------------------------------
// The reference divides through its own reciprocal:
//   Q = BigInt(BigFloat::mul(BigFloat(a), BigFloat(b).reciprocal(n_a + 16), n_a + 16), mode);
//   R = a - Q * b;
//   one adjustment by +-1 when R breaks the mode's bound (check = true).
// Replayed step by step on the device like the reciprocal: the estimate, Q * b
// and the exact sums and differences are device kernels; the host follows
// lengths, point positions and signs, and reads one compare word per test.

enum DivMode : uint32_t { kTruncate = 0, kFloor = 1, kCeil = 2, kRoundHalfUp = 3 };

// sign(|a| - |b|) of two integer values (point positions <= 0).
int cmp_abs(const DVal& a, const DVal& b, int* out) {
    if (a.zero() || b.zero()) {
        *out = a.zero() ? (b.zero() ? 0 : -1) : 1;
        return BGPU_OK;
    }
    const int64_t pp = std::max(a.pp - (int64_t)a.tz, b.pp - (int64_t)b.tz);
    const int64_t len = std::max((int64_t)a.n - a.pp, (int64_t)b.n - b.pp) + pp;
    if (len <= 0 || len >= ((int64_t)1 << 31)) return BGPU_ERR_CAPACITY;
    FrameOp f{a.d, pp - a.pp, (uint32_t)a.n, b.d, pp - b.pp, (uint32_t)b.n, (uint32_t)len, 0, nullptr};
    unsigned long long* dr = nullptr;
    int rc = result_block(&dr);
    if (rc == BGPU_OK) rc = cuda_status(launch_frame_cmp(f, dr, g.stream));
    unsigned long long w = 0;
    if (rc == BGPU_OK) rc = read_back(reinterpret_cast<const uint32_t*>(dr), reinterpret_cast<uint32_t*>(&w), 2);
    if (rc != BGPU_OK) return rc;
    *out = w == 0 ? 0 : ((w & 3u) == 1u ? 1 : -1);
    return BGPU_OK;
}

// The exact product of two integer values into `slot`.
int int_product(const DVal& a, const DVal& b, int slot, DVal* out) {
    if (a.zero() || b.zero()) {
        *out = DVal{};
        return BGPU_OK;
    }
    const size_t nres = a.n + b.n + 1;
    if (nres > ((size_t)1 << 31)) return BGPU_ERR_CAPACITY;
    int rc;
    uint32_t* dres = rslot(slot, nres, &rc);
    unsigned long long* dr = nullptr;
    if (rc == BGPU_OK) rc = digits_product(a, 0, b, 0, dres, nres);
    if (rc == BGPU_OK) rc = result_block(&dr);
    uint32_t r[4];
    if (rc == BGPU_OK) rc = extent(dr, dres, nres, 0, 0, r);
    if (rc != BGPU_OK) return rc;
    if (r[0] == 0 || r[1] >= r[0]) return BGPU_ERR_CUDA;  // a product of nonzero values is nonzero
    *out = DVal{dres + r[1], r[0] - r[1], a.pp + b.pp - (int64_t)r[1], a.neg != b.neg, 0, r[3], slot};
    return BGPU_OK;
}

// BigInt(const BigFloat&, mode) (src/bigint.cpp:1142-1147, convert_from_BigFloat
// :1156-1172, _round :1072-1110) of the estimate P, whose bottom digit is
// nonzero (BigFloat::mul removes tail zeros).  Digits below the point are
// dropped; Floor and Ceil raise |Q| by one when the sign asks for it (a
// dropped digit is always nonzero here), RoundHalfUp when the top dropped bit
// is set.  When every digit lies below the point and none is added, the
// reference is left with an empty digit vector (undefined behaviour, reached
// for 2^-28 <= |P| < 1); the engine returns the value that truncation means,
// zero.
int estimate_to_int(const DVal& p, uint32_t mode, const DVal& one_pos, const DVal& one_neg, DVal* q) {
    if (p.zero() || p.pp > (int64_t)p.n) {
        *q = DVal{};
        return BGPU_OK;
    }
    if (p.pp <= 0) {  // an integer already: -pp zero digits below
        *q = p;
        return BGPU_OK;
    }
    const size_t k = (size_t)p.pp;  // dropped digits d[0..k)
    bool inc = false;
    if (mode == kFloor) {
        inc = p.neg;
    } else if (mode == kCeil) {
        inc = !p.neg;
    } else if (mode == kRoundHalfUp) {
        uint32_t top_dropped = 0;
        const int rc = read_back(p.d + (k - 1), &top_dropped, 1);
        if (rc != BGPU_OK) return rc;
        inc = (top_dropped >> 27) != 0;
    }
    if (k == p.n) {  // nothing above the point
        *q = inc ? (p.neg ? one_neg : one_pos) : DVal{};
        return BGPU_OK;
    }
    const DVal kept{p.d + k, p.n - k, 0, p.neg, 0, p.top, p.slot};
    if (!inc) {
        *q = kept;
        return BGPU_OK;
    }
    return add_or_sub(kept, p.neg ? one_neg : one_pos, false, kRsDivQ, q);  // |Q| + 1
}

// An integer value as Digits (zero: {0}) into a host buffer.
int int_out(const DVal& v, uint32_t* out, size_t cap, size_t* len, int* neg) {
    if (v.zero()) {
        *len = 1;
        *neg = 0;
        if (cap < 1) return BGPU_ERR_OUT_CAPACITY;
        out[0] = 0;
        return BGPU_OK;
    }
    if (v.pp > 0) return BGPU_ERR_CUDA;  // not an integer
    const size_t low = (size_t)(-v.pp);
    *len = v.n + low;
    *neg = v.neg ? 1 : 0;
    if (*len > cap) return BGPU_ERR_OUT_CAPACITY;
    if (low) memset(out, 0, low * 4);
    return device_to_host(out + low, v.d, v.n * 4, g.stream);
}

// A host integer (Digits, no leading zeros) on the device as BigFloat(x): tail
// zeros removed, point position -tz.
int upload_int(int slot, const uint32_t* digits, size_t n, bool neg, DVal* out) {
    if (n == 1 && digits[0] == 0) {
        *out = DVal{};
        return BGPU_OK;
    }
    size_t tz = 0;
    while (digits[tz] == 0) ++tz;
    int rc;
    uint32_t* d = rslot(slot, n - tz, &rc);
    if (rc == BGPU_OK) rc = host_to_device(d, digits + tz, (n - tz) * 4, g.stream, nullptr);
    if (rc != BGPU_OK) return rc;
    *out = DVal{d, n - tz, -(int64_t)tz, neg, 0, digits[n - 1], slot};
    return BGPU_OK;
}

int divmod_steps(const uint32_t* a, size_t na, bool a_neg, const uint32_t* b, size_t nb, bool b_neg,
                 uint32_t mode, bool check, uint32_t* q, size_t q_cap, size_t* q_len, int* q_neg,
                 uint32_t* r, size_t r_cap, size_t* r_len, int* r_neg) {
    for (const auto& [d, n] : {std::pair{a, na}, std::pair{b, nb}}) {
        if (n >= ((size_t)1 << 31)) return BGPU_ERR_CAPACITY;
        for (size_t i = 0; i < n; ++i)
            if (d[i] >> 28) return BGPU_ERR_INVALID_ARG;
        if (n > 1 && d[n - 1] == 0) return BGPU_ERR_INVALID_ARG;  // a leading zero digit
    }
    if (nb == 1 && b[0] == 0) return BGPU_ERR_INVALID_ARG;  // division by zero (std::domain_error)
    if (mode > kRoundHalfUp) mode = kTruncate;            // the reference's default branch
    DVal A, B, Q, R;
    int rc = upload_int(kRsDivA, a, na, a_neg && !(na == 1 && a[0] == 0), &A);
    if (rc == BGPU_OK) rc = upload_int(kRsDivB, b, nb, b_neg, &B);
    if (rc != BGPU_OK) return rc;
    if (!A.zero()) {
        const size_t precision = na + 16;  // PROTECT_PRECISION
        DVal inv, p, one_pos, one_neg, qb;
        rc = reciprocal_val(B, precision, &inv);
        if (rc == BGPU_OK) rc = mul_trunc(A, inv, precision, kRsDivP, &p);
        if (rc == BGPU_OK) rc = upload_digits(kRsOne, std::vector<uint32_t>{1u}, 0, false, &one_pos);
        if (rc != BGPU_OK) return rc;
        one_neg = one_pos;
        one_neg.neg = true;
        rc = estimate_to_int(p, mode, one_pos, one_neg, &Q);
        if (rc == BGPU_OK) rc = int_product(Q, B, kRsDivQB, &qb);
        if (rc == BGPU_OK) rc = add_or_sub(A, qb, true, kRsDivR, &R);  // R = a - Q * b
        if (rc != BGPU_OK) return rc;
        if (check && !R.zero()) {
            bool adjust;
            int c = 0;
            if (mode == kRoundHalfUp) {
                DVal r2;
                rc = add_or_sub(R, R, false, kRsDivR2, &r2);
                if (rc == BGPU_OK) rc = cmp_abs(r2, B, &c);
                adjust = c > 0 || (c == 0 && R.neg == a_neg);
            } else {
                rc = cmp_abs(R, B, &c);
                const bool over = c >= 0;
                if (mode == kFloor) adjust = (R.neg != b_neg) || over;
                else if (mode == kCeil) adjust = (R.neg == b_neg) || over;
                else adjust = (R.neg != a_neg) || over;
            }
            if (rc != BGPU_OK) return rc;
            if (adjust) {
                DVal q2, r2;
                const bool down = R.neg != b_neg;  // R += b, --Q; else R -= b, ++Q
                rc = add_or_sub(R, B, !down, kRsDivR2, &r2);
                if (rc == BGPU_OK) rc = add_or_sub(Q, one_pos, down, kRsDivQ2, &q2);
                if (rc != BGPU_OK) return rc;
                Q = q2;
                R = r2;
            }
        }
    }
    const int rq = int_out(Q, q, q_cap, q_len, q_neg);
    if (rq != BGPU_OK && rq != BGPU_ERR_OUT_CAPACITY) return rq;
    const int rr = int_out(R, r, r_cap, r_len, r_neg);
    if (rr != BGPU_OK && rr != BGPU_ERR_OUT_CAPACITY) return rr;
    rc = check_device_error(BGPU_OK);
    if (rc != BGPU_OK) return rc;
    return rq != BGPU_OK ? rq : rr;
}

}  // namespace

Tuning& tuning() { return g_tuning; }

}  // namespace bgpu

using namespace bgpu;

extern "C" {

int bgpu_init(int device) {
    std::lock_guard<std::mutex> lk(g_mu);
    return init_locked(device);
}

int bgpu_shutdown(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    release_locked();
    return BGPU_OK;
}

const char* bgpu_strerror(int code) {
    switch (code) {
        case BGPU_OK: return "ok";
        case BGPU_ERR_INVALID_ARG: return "invalid argument";
        case BGPU_ERR_NO_DEVICE: return "no usable CUDA device";
        case BGPU_ERR_OOM: return "out of memory";
        case BGPU_ERR_CAPACITY: return "product exceeds the largest supported transform";
        case BGPU_ERR_OUT_CAPACITY: return "output buffer too small";
        case BGPU_ERR_CUDA: return "CUDA error";
        case BGPU_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
        case BGPU_ERR_NOT_INIT: return "engine not initialized (call bgpu_init)";
        default: return "unknown status";
    }
}

int bgpu_mul_u64(const uint64_t* a, size_t na, const uint64_t* b, size_t nb, uint64_t* out,
                 size_t out_cap, size_t* out_len, uint32_t flags, bgpu_stats* stats) {
    if (!a || !b || !out_len || (!out && out_cap) || na == 0 || nb == 0) return BGPU_ERR_INVALID_ARG;
    if (!valid_method(flags, true)) return BGPU_ERR_INVALID_ARG;
    const uint32_t fb = (flags >> 8) & 0x1Fu;
    if (fb && (fb < 8 || fb > 20)) return BGPU_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_mu);
    if (g.device < 0) return BGPU_ERR_NOT_INIT;
    cudaSetDevice(g.device);
    return mul_u64_locked(a, na, b, nb, out, out_cap, out_len, flags, stats);
}

int bgpu_mul_digits(const uint32_t* a, size_t na, const uint32_t* b, size_t nb,
                    size_t output_precision, int64_t* point_pos, uint32_t* out, size_t out_cap,
                    size_t* out_len, uint32_t flags, bgpu_stats* stats) {
    if (!a || !b || !out_len || (!out && out_cap) || na == 0 || nb == 0) return BGPU_ERR_INVALID_ARG;
    if (!valid_method(flags, false)) return BGPU_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_mu);
    if (g.device < 0) return BGPU_ERR_NOT_INIT;
    cudaSetDevice(g.device);
    return mul_digits_locked(a, na, b, nb, output_precision, point_pos, out, out_cap, out_len,
                             flags, stats);
}

int bgpu_reciprocal_digits(const uint32_t* digits, size_t n, int64_t point_pos, int is_neg,
                           size_t precision, uint32_t* out, size_t out_cap, size_t* out_len,
                           int64_t* out_point_pos, int* out_is_neg) {
    if (!digits || n == 0 || !out_len || !out_point_pos || !out_is_neg || (!out && out_cap))
        return BGPU_ERR_INVALID_ARG;
    if (point_pos > BGPU_MAX_POINT_POS || point_pos < -BGPU_MAX_POINT_POS) return BGPU_ERR_CAPACITY;
    std::lock_guard<std::mutex> lk(g_mu);
    if (g.device < 0) return BGPU_ERR_NOT_INIT;
    cudaSetDevice(g.device);
    return reciprocal_locked(digits, n, point_pos, is_neg != 0, precision, out, out_cap, out_len,
                             out_point_pos, out_is_neg);
}

int bgpu_divmod_digits(const uint32_t* a, size_t na, int a_neg, const uint32_t* b, size_t nb, int b_neg,
                       uint32_t mode, int check, uint32_t* q, size_t q_cap, size_t* q_len, int* q_neg,
                       uint32_t* r, size_t r_cap, size_t* r_len, int* r_neg) {
    if (!a || !b || na == 0 || nb == 0 || !q_len || !q_neg || !r_len || !r_neg || (!q && q_cap) ||
        (!r && r_cap) || mode > 255)
        return BGPU_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_mu);
    if (g.device < 0) return BGPU_ERR_NOT_INIT;
    cudaSetDevice(g.device);
    return with_device_status(divmod_steps(a, na, a_neg != 0, b, nb, b_neg != 0, mode, check != 0, q, q_cap,
                                           q_len, q_neg, r, r_cap, r_len, r_neg));
}

int bgpu_selftest_wait(uint32_t spin_limit, int set_flag) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (g.device < 0) return BGPU_ERR_NOT_INIT;
    cudaSetDevice(g.device);
    // one flag word in the grow-only I/O buffer: 0 (no epoch) or epoch 1 set
    int rc = ensure(&g.d_io, &g.io_bytes, 256);
    if (rc != BGPU_OK) return rc;
    uint64_t* flag = static_cast<uint64_t*>(g.d_io);
    const uint64_t word = set_flag ? ((uint64_t)1 << 4) | (2u << 2) : 0;
    cudaError_t e = cudaMemcpyAsync(flag, &word, sizeof(word), cudaMemcpyHostToDevice, g.stream);
    if (e == cudaSuccess) e = launch_wait_selftest(flag, 1, spin_limit, g.d_err, g.stream);
    if (e != cudaSuccess) return cuda_status(e);
    return check_device_error(BGPU_OK);
}

int bgpu_mul_u64_many(const bgpu_host_product* products, size_t count, uint32_t flags) {
    if (!products && count) return BGPU_ERR_INVALID_ARG;
    if (!valid_method(flags, false)) return BGPU_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_mu);
    if (g.device < 0) return BGPU_ERR_NOT_INIT;
    cudaSetDevice(g.device);
    return mul_u64_many_locked(products, count, flags);
}

int bgpu_pow_u64(const uint64_t* base, size_t nbase, uint32_t exponent, uint64_t* out,
                 size_t out_cap, size_t* out_len) {
    if (!base || !out_len || (!out && out_cap) || nbase == 0) return BGPU_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_mu);
    if (g.device < 0) return BGPU_ERR_NOT_INIT;
    cudaSetDevice(g.device);
    return pow_u64_locked(base, nbase, exponent, out, out_cap, out_len);
}

int bgpu_mul_u64_device(const uint64_t* d_a, size_t na, const uint64_t* d_b, size_t nb,
                        uint64_t* d_out, uint32_t flags, void* stream) {
    if (!d_a || !d_b || !d_out || na == 0 || nb == 0) return BGPU_ERR_INVALID_ARG;
    if (!valid_method(flags, false)) return BGPU_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_mu);
    if (g.device < 0) return BGPU_ERR_NOT_INIT;
    cudaSetDevice(g.device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);  // 0 = the legacy default stream
    const bool square = (d_a == d_b && na == nb);
    // A promised-independent product overlaps the previous one's tail unless
    // its operands overlap the previous call's output on this stream.
    auto hits_prev = [&](const uint64_t* p, size_t n) {
        const char* lo = reinterpret_cast<const char*>(p);
        const char* plo = static_cast<const char*>(g.prev_out);
        return lo < plo + g.prev_out_bytes && plo < lo + n * 8;
    };
    const bool overlap = (flags & BGPU_INDEPENDENT) &&
                         !(st == g.prev_stream && (hits_prev(d_a, na) || hits_prev(d_b, nb)));
    g.prev_stream = st;
    g.prev_out = d_out;
    g.prev_out_bytes = (na + nb) * 8;
    if (const uint32_t sm = small_method(flags, na, nb)) {
        g.last_launches = 1;
        return launch_small(sm, d_a, na, d_b, nb, d_out, st);
    }
    if (na + nb > ((size_t)1 << 31)) return BGPU_ERR_CAPACITY;
    if (beyond_transform(na, nb)) return huge_product(d_a, na, d_b, nb, d_out, square, st);
    OperandDesc oa{d_a, (uint32_t)na, (uint32_t)(2 * na), kFmtLimb64};
    OperandDesc ob{d_b, (uint32_t)nb, (uint32_t)(2 * nb), kFmtLimb64};
    return multiply_device(oa, ob, square, d_out, kFmtLimb64, na + nb, flags, st, nullptr, overlap);
}

int bgpu_device_status(void* stream) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (g.device < 0) return BGPU_ERR_NOT_INIT;
    cudaSetDevice(g.device);
    cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_status(e);
    return check_device_error(BGPU_OK);
}

uint32_t bgpu_last_launch_count(void) { return g.last_launches; }

static EngineHooks hooks_locked() {
    EngineHooks h{};
    for (int ps = 0; ps < kNumSets; ++ps) h.consts[ps] = g.consts[ps];
    h.err = g.d_err;
    return h;
}

// Limbs of V_k and its offset in the reciprocal cache.
static uint64_t pow_mk(int k) { return ((uint64_t)1 << k) + (((uint64_t)1 << k) >> 6) + 2; }
static uint64_t pow_voff(int k) {
    uint64_t o = 0;
    for (int i = 0; i < k; ++i) o += pow_mk(i);
    return o;
}

// Grows a device buffer to `need` bytes keeping its first `keep` bytes.
static int grow_keep(uint64_t** p, size_t* bytes, size_t need, size_t keep, cudaStream_t st) {
    if (*bytes >= need) return BGPU_OK;
    void* np = nullptr;
    if (cudaMalloc(&np, need) != cudaSuccess) {
        cudaGetLastError();
        return BGPU_ERR_OOM;
    }
    cudaError_t e = cudaSuccess;
    if (*p && keep) e = cudaMemcpyAsync(np, *p, keep, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaFree(np);
        return cuda_status(e);
    }
    cudaFree(*p);
    *p = static_cast<uint64_t*>(np);
    *bytes = need;
    return BGPU_OK;
}

// Q_0 .. Q_(J-1) (and with_v: V_0 .. V_(J-1)) in the engine's cache, computed
// on the device the first time a size needs them; later calls of the same or
// smaller size reuse them, as the reference keeps its powers of ten
// (get_pow_of_ten, src/bigint.cpp:154-173).  The reciprocals are a chain:
// V_k^2 <= V_(k+1) (both floors of the same real, squared), one Newton step
// from below brings it within a few units, and single correction steps
// (r >= Q: r -= Q, V += 1) make it exact.
static int ensure_powers(int J, bool with_v, cudaStream_t st, uint32_t* nl) {
    if (J <= 0) return BGPU_OK;
    if (g.pq_levels < J) {
        const int have = g.pq_levels;
        int rc = grow_keep(&g.d_pq, &g.pq_bytes, ((size_t)1 << J) * 8,
                           have ? (((size_t)1 << have) - 1) * 8 : 0, st);
        if (rc != BGPU_OK) return rc;
        if (have == 0) {
            const uint64_t ten19 = 10000000000000000000ull;
            cudaError_t e = cudaMemcpyAsync(g.d_pq, &ten19, 8, cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return cuda_status(e);
        }
        for (int k = std::max(have, 1) - 1; k + 1 < J; ++k) {  // Q_(k+1) = Q_k^2
            const uint64_t w = (uint64_t)1 << k;
            rc = device_product(g.d_pq + (w - 1), w, g.d_pq + (w - 1), w, g.d_pq + (2 * w - 1), st, nl);
            if (rc != BGPU_OK) return rc;
        }
        g.pq_levels = J;
    }
    if (!with_v || g.pv_levels >= J) return BGPU_OK;
    const int have = g.pv_levels;
    int rc = grow_keep(&g.d_pv, &g.pv_bytes, pow_voff(J) * 8 + 64, pow_voff(have) * 8, st);
    if (rc != BGPU_OK) return rc;
    if (have == 0) {  // V_0 = floor(2^128 / 10^19)
        const unsigned __int128 v0 = ~(unsigned __int128)0 / 10000000000000000000ull;
        std::vector<uint64_t> hv(pow_mk(0), 0);
        hv[0] = (uint64_t)v0;
        hv[1] = (uint64_t)(v0 >> 64);
        cudaError_t e = cudaMemcpyAsync(g.d_pv, hv.data(), hv.size() * 8, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_status(e);
        g.pv_levels = 1;
        if (J == 1) return BGPU_OK;
    }
    // scratch of the largest step (K = 2^(J-1)): X, P, R, D, the constant 1, a
    // flag and the carry-scan words
    const uint64_t Kmax = (uint64_t)1 << (J - 1);
    const uint64_t mmax = pow_mk(J - 2 < 0 ? 0 : J - 2);
    const uint64_t nacc = accumulate_blocks(2 * Kmax + 2);
    const uint64_t scratch = 6 * mmax + Kmax + 4 * Kmax + 64 + 8 + nacc + 64;
    uint64_t* xs = nullptr;
    if (cudaMalloc(reinterpret_cast<void**>(&xs), scratch * 8) != cudaSuccess) {
        cudaGetLastError();
        return BGPU_ERR_OOM;
    }
    uint64_t* one = xs + scratch - nacc - 16;
    uint32_t* flag = reinterpret_cast<uint32_t*>(one + 1);
    uint32_t* agg = reinterpret_cast<uint32_t*>(one + 8);
    uint32_t* cin = agg + nacc;
    const uint64_t c1 = 1;
    cudaError_t e = cudaMemcpyAsync(one, &c1, 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    rc = cuda_status(e);
    for (int k = g.pv_levels - 1; rc == BGPU_OK && k + 1 < J; ++k) {
        const uint64_t K = (uint64_t)1 << (k + 1), el = 2 * K, m = pow_mk(k), m1 = pow_mk(k + 1);
        const uint64_t* q = g.d_pq + (K - 1);
        const uint64_t* v = g.d_pv + pow_voff(k);
        uint64_t* v1 = g.d_pv + pow_voff(k + 1);
        uint64_t* X = xs;                 // 2m
        uint64_t* P = X + 2 * m + 8;      // K + 2m
        uint64_t* R = P + K + 2 * m + 8;  // el + 1
        uint64_t* Dd = R + el + 8;        // 2m + el + 1
        rc = device_product(v, m, v, m, X, st, nl);  // X = V_k^2 <= V_(k+1)
        if (rc == BGPU_OK) rc = device_product(q, K, X, 2 * m, P, st, nl);  // P = Q X < 2^(64 el)
        if (rc == BGPU_OK) rc = cuda_status(launch_not_limbs(P, (uint32_t)el, R, st));
        if (rc == BGPU_OK) rc = cuda_status(launch_accumulate(R, el + 1, one, 1, agg, cin, st));
        if (rc == BGPU_OK) rc = device_product(X, 2 * m, R, el + 1, Dd, st, nl);  // X (2^E - Q X)
        // V' = X + floor(X R / 2^E): Newton from below, within a few units of V_(k+1)
        if (rc == BGPU_OK) rc = cuda_status(cudaMemsetAsync(v1, 0, m1 * 8, st));
        if (rc == BGPU_OK)
            rc = cuda_status(cudaMemcpyAsync(v1, X, std::min(2 * m, m1) * 8, cudaMemcpyDeviceToDevice, st));
        if (rc == BGPU_OK)
            rc = cuda_status(launch_accumulate(v1, m1, Dd + el, std::min<uint64_t>(2 * m + 1, m1), agg, cin, st));
        // exact: R = 2^E - Q V' (>= 0); while R >= Q: R -= Q, V' += 1
        if (rc == BGPU_OK) rc = device_product(q, K, v1, m1, P, st, nl);
        if (rc == BGPU_OK) rc = cuda_status(launch_not_limbs(P, (uint32_t)el, R, st));
        if (rc == BGPU_OK) rc = cuda_status(launch_accumulate(R, el + 1, one, 1, agg, cin, st));
        for (int it = 0; rc == BGPU_OK; ++it) {
            if (it == 64) {  // the Newton step is within a few units
                rc = BGPU_ERR_CUDA;
                break;
            }
            uint32_t f = 0;
            rc = cuda_status(launch_fix_step(R, (uint32_t)(el + 1), q, (uint32_t)K, v1, (uint32_t)m1, flag, st));
            if (rc == BGPU_OK) rc = read_back(flag, &f, 1);
            if (!f) break;
        }
        if (rc == BGPU_OK) g.pv_levels = k + 2;
    }
    cudaStreamSynchronize(st);
    cudaFree(xs);
    return rc;
}

// A batch of equal-size device products on `st` (the levels of the decimal
// conversions): schoolbook or Karatsuba classes as one launch over a
// descriptor array, up to 128 transform-size products as direct launches,
// more through a batch plan.
static int run_products(const bgpu_product* pr, size_t count, cudaStream_t st, uint32_t* launches) {
    if (count == 0) return BGPU_OK;
    const size_t na = pr[0].na, nb = pr[0].nb;
    const Tuning& tu = tuning();
    const bool school = na + nb <= tu.batch_schoolbook_max_limbs;
    if (school || (na + nb <= tu.batch_karatsuba_max_limbs && karatsuba_fits(na, nb))) {
        std::vector<SchoolDesc> d(count);
        for (size_t i = 0; i < count; ++i)
            d[i] = SchoolDesc{pr[i].a, pr[i].b, pr[i].out, (uint32_t)pr[i].na, (uint32_t)pr[i].nb};
        int rc = ensure(&g.d_desc, &g.desc_bytes, count * sizeof(SchoolDesc));
        if (rc != BGPU_OK) return rc;
        cudaError_t e = cudaMemcpyAsync(g.d_desc, d.data(), count * sizeof(SchoolDesc), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // d goes out of scope
        const SchoolDesc* dd = static_cast<const SchoolDesc*>(g.d_desc);
        if (e == cudaSuccess)
            e = school ? launch_schoolbook_batch(dd, (uint32_t)count, st) : launch_karatsuba_batch(dd, (uint32_t)count, st);
        *launches += 1;
        return cuda_status(e);
    }
    if (count <= 128) {
        for (size_t i = 0; i < count; ++i) {
            const int rc = device_product(pr[i].a, pr[i].na, pr[i].b, pr[i].nb, pr[i].out, st, launches);
            if (rc != BGPU_OK) return rc;
        }
        return BGPU_OK;
    }
    bgpu_batch_plan_s* plan = nullptr;
    int rc = batch_plan_create(pr, count, BGPU_METHOD_AUTO, g.device, hooks_locked(), &plan);
    if (rc != BGPU_OK) return rc;
    rc = batch_plan_run(plan, st);
    if (rc == BGPU_OK) rc = cuda_status(cudaStreamSynchronize(st));
    *launches += batch_plan_launches(plan);
    batch_plan_destroy(plan);
    return rc;
}

// Decimal text to Digits: BigInt(const std::string&) with hex = false
// (src/bigint.cpp:25-90) and convert_from_dec_string (:92-124).  The sign and
// the digit characters are picked out on the host exactly as the reference
// reads them; the value is built on the device (decimal.cu): leaves of 19
// digits, then levels of hi * 10^(19 * 2^j) + lo, each level one batch plan
// of equal products and one segmented carry add.
static int from_decimal_locked(const char* s, size_t len, uint32_t* out, size_t out_cap, size_t* out_len,
                               int* out_neg) {
    size_t i = 0;
    bool neg = false;
    for (; i < len; ++i) {  // before the first digit, any '-' makes the number negative
        const unsigned char c = (unsigned char)s[i];
        if (c >= '0' && c <= '9') break;
        if (c == '-') neg = true;
    }
    std::vector<uint8_t> dig;
    dig.reserve(len - i);
    for (; i < len; ++i) {  // other characters are skipped; leading zeros dropped
        const unsigned char c = (unsigned char)s[i];
        if (c < '0' || c > '9' || (dig.empty() && c == '0')) continue;
        dig.push_back((uint8_t)(c - '0'));
    }
    const uint64_t D = dig.size();
    if (D == 0) {  // the reference's zero: one digit 0, not negative
        *out_len = 1;
        *out_neg = 0;
        if (out_cap < 1) return BGPU_ERR_OUT_CAPACITY;
        out[0] = 0;
        return BGPU_OK;
    }
    const uint64_t leaves = (D + 18) / 19;
    const int J = ceil_log2(leaves);
    if (J > 25) return BGPU_ERR_CAPACITY;  // the top level's product is the largest general transform
    const uint64_t NL = (uint64_t)1 << J;  // limbs of every level
    const uint32_t w0 = (uint32_t)std::min<uint64_t>(kParseLeafLimbs, NL);  // limbs of a leaf built per thread
    int j0 = 0;
    while ((1u << j0) < w0) ++j0;
    const uint64_t nd = (64 * NL + 27) / 28;  // Digits of the result, before stripping
    const size_t dig_off = 0, lvl_off = align256(D), o_off = lvl_off + 2 * align256(NL * 8);
    const size_t acc_off = o_off + align256(nd * 4);
    const size_t acc_words = accumulate_blocks(NL) + 64;
    int rc = ensure(&g.d_dec, &g.dec_bytes, acc_off + 2 * acc_words * 4);
    if (rc != BGPU_OK) return rc;
    char* base = static_cast<char*>(g.d_dec);
    uint8_t* ddig = reinterpret_cast<uint8_t*>(base + dig_off);
    uint64_t* lvl[2] = {reinterpret_cast<uint64_t*>(base + lvl_off),
                        reinterpret_cast<uint64_t*>(base + lvl_off + align256(NL * 8))};
    uint32_t* dout = reinterpret_cast<uint32_t*>(base + o_off);
    cudaStream_t st = g.stream;
    rc = host_to_device(ddig, dig.data(), D, st, nullptr);
    if (rc != BGPU_OK) return rc;
    uint32_t nl = 0;
    rc = ensure_powers(J, false, st, &nl);  // 10^(19 * 2^j) at limb 2^j - 1, 2^j limbs
    if (rc != BGPU_OK) return rc;
    const uint64_t* q = g.d_pq;
    uint32_t* agg = reinterpret_cast<uint32_t*>(base + acc_off);
    uint32_t* cin = agg + acc_words;
    // Only segments holding digits are built: the levels are 2^J limbs wide but
    // the number may fill little more than half of them.  Everything above is
    // zero from the start, and what a level leaves of the level two below
    // lies inside the region it overwrites (its segments are coarser).
    cudaError_t e = cudaMemsetAsync(lvl[0], 0, NL * 8, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(lvl[1], 0, NL * 8, st);
    if (e == cudaSuccess) e = launch_dec_leaves(ddig, D, w0, (leaves + w0 - 1) / w0, lvl[0], st);
    if (e != cudaSuccess) return cuda_status(e);
    int cur = 0;
    std::vector<bgpu_product> prods;
    for (int j = j0; j < J; ++j) {
        const uint64_t w1 = (uint64_t)1 << j, pairs = (leaves + 2 * w1 - 1) / (2 * w1);
        prods.resize(pairs);
        for (uint64_t p = 0; p < pairs; ++p)
            prods[p] = bgpu_product{lvl[cur] + (2 * p + 1) * w1, w1, q + (w1 - 1), w1, lvl[cur ^ 1] + p * 2 * w1};
        rc = run_products(prods.data(), pairs, st, &nl);
        if (rc != BGPU_OK) return rc;
        if (pairs <= 8 && w1 >= 4096) {  // few long segments: one multi-block carry scan each
            for (uint64_t p = 0; p < pairs && e == cudaSuccess; ++p)
                e = launch_accumulate(lvl[cur ^ 1] + p * 2 * w1, 2 * w1, lvl[cur] + 2 * p * w1, w1, agg, cin, st);
        } else {
            e = launch_seg_add_low(lvl[cur ^ 1], lvl[cur], (uint32_t)w1, pairs, st);
        }
        if (e != cudaSuccess) return cuda_status(e);
        cur ^= 1;
    }
    e = launch_limbs_to_digits28(lvl[cur], (uint32_t)NL, dout, (uint32_t)nd, st);
    if (e != cudaSuccess) return cuda_status(e);
    std::vector<uint32_t> h(nd);
    rc = device_to_host(h.data(), dout, nd * 4, st);
    rc = check_device_error(rc);
    if (rc != BGPU_OK) return rc;
    const size_t n = strip32(h.data(), nd);
    *out_len = n;
    *out_neg = neg ? 1 : 0;
    if (n > out_cap) return BGPU_ERR_OUT_CAPACITY;
    memcpy(out, h.data(), n * 4);
    g.last_launches = nl;
    return BGPU_OK;
}

// BigInt to decimal text: BigInt::print (src/bigint.cpp:175-247), the
// reference's print_dec divide and conquer, on the device (decimal.cu).  The
// value is split top-down into halves by Q_k = 10^(19 * 2^k): a level-j
// segment s < Q_(j-1)^2 becomes s mod Q_(j-1) and s div Q_(j-1), the quotient
// estimated with the exact reciprocal V_(j-1) = floor(2^(128 * 2^(j-1)) / Q_(j-1))
// (two batched products per level) and corrected once per segment on the
// device.  The reciprocals are a chain: V_k^2 is at most V_(k+1) (both are
// floors of the same real, squared), one Newton step from below brings it
// within a few units, and single correction steps make it exact.  Leaves of
// kPrintLeafLimbs limbs print 19 * kPrintLeafLimbs characters per thread.

// Decimal text (no sign, no leading zeros) of the integer whose Digits are n
// digits at hsrc (host) or dsrc (device), the top one `top` (nonzero), above
// `low` zero digits: h[first..) on return.
static int dec_chars(const uint32_t* hsrc, const uint32_t* dsrc, size_t low, size_t n, uint32_t top,
                     std::vector<char>* hv, size_t* first_out) {
    std::vector<char>& h = *hv;
    if (n == 0) {
        h.assign(1, '0');
        *first_out = 0;
        return BGPU_OK;
    }
    const size_t nsrc = n;
    n += low;
    const uint64_t bits = 28 * (uint64_t)(n - 1) + (32 - __builtin_clz(top));
    const uint64_t dmax = (uint64_t)std::ceil((double)bits * 0.30102999566398120) + 1;  // >= decimal digits
    const int J = ceil_log2((dmax + 18) / 19);
    if (J > 25) return BGPU_ERR_CAPACITY;
    const uint64_t NL = (uint64_t)1 << J;
    const uint32_t w0 = (uint32_t)std::min<uint64_t>(kPrintLeafLimbs, NL);  // limbs per printed leaf
    int jleaf = 0;
    while ((1u << jleaf) < w0) ++jleaf;
    auto mk = pow_mk;
    // arena (limbs)
    uint64_t off = 0;
    auto take = [&](uint64_t limbs) {
        const uint64_t o = off;
        off += (limbs + 31) & ~(uint64_t)31;
        return o;
    };
    const uint64_t o_lvl0 = take(NL), o_lvl1 = take(NL), o_t = take(2 * NL + 4 * J + 64), o_u = take(NL);
    const uint64_t o_dig = take((n + 1) / 2 + 1), o_chr = take((19 * NL + 7) / 8 + 1);
    int rc = ensure(&g.d_dec, &g.dec_bytes, off * 8);
    if (rc != BGPU_OK) return rc;
    uint64_t* A = static_cast<uint64_t*>(g.d_dec);
    uint64_t* lvl[2] = {A + o_lvl0, A + o_lvl1};
    uint64_t* tb = A + o_t;
    uint64_t* ub = A + o_u;
    uint32_t* ddig = reinterpret_cast<uint32_t*>(A + o_dig);
    char* chars = reinterpret_cast<char*>(A + o_chr);
    cudaStream_t st = g.stream;

    // the value, as NL limbs; the powers of ten and their reciprocals
    cudaError_t e = low ? cudaMemsetAsync(ddig, 0, low * 4, st) : cudaSuccess;
    rc = cuda_status(e);
    if (rc == BGPU_OK)
        rc = hsrc ? host_to_device(ddig + low, hsrc, nsrc * 4, st, nullptr)
                  : cuda_status(cudaMemcpyAsync(ddig + low, dsrc, nsrc * 4, cudaMemcpyDeviceToDevice, st));
    if (rc != BGPU_OK) return rc;
    e = launch_digits28_to_limbs(ddig, (uint32_t)n, lvl[0], (uint32_t)NL, st);
    if (e != cudaSuccess) return cuda_status(e);
    uint32_t nl = 0;
    rc = ensure_powers(J, J > jleaf, st, &nl);
    if (rc != BGPU_OK) return rc;
    const uint64_t* qp = g.d_pq;
    const uint64_t* vp = g.d_pv;
    // top-down division levels
    int cur = 0;
    std::vector<bgpu_product> prods;
    for (int j = J; j > jleaf; --j) {
        // segments above the value's last decimal digit are zero: their halves
        // are never read (the level below reads only its own, finer, active part)
        const uint64_t w = (uint64_t)1 << (j - 1), m = mk(j - 1), ts = 2 * w + m;
        const uint64_t count = std::min<uint64_t>(NL >> j, (dmax + 19 * 2 * w - 1) / (19 * 2 * w));
        const uint64_t* q = qp + (w - 1);
        const uint64_t* v = vp + pow_voff(j - 1);
        for (int pass = 0; pass < 2; ++pass) {
            prods.resize(count);
            for (uint64_t p = 0; p < count; ++p)
                prods[p] = pass == 0
                               ? bgpu_product{lvl[cur] + 2 * w * p, 2 * w, v, m, tb + ts * p}
                               : bgpu_product{tb + ts * p + 2 * w, w, q, w, ub + 2 * w * p};
            rc = run_products(prods.data(), count, st, &nl);
            if (rc != BGPU_OK) return rc;
        }
        e = launch_seg_divstep(lvl[cur], ub, tb, (uint32_t)ts, q, (uint32_t)w, count, lvl[cur ^ 1], st);
        if (e != cudaSuccess) return cuda_status(e);
        cur ^= 1;
    }
    const uint64_t nleaf = std::min<uint64_t>(NL / w0, (dmax + 19 * w0 - 1) / (19 * w0));
    e = launch_dec_print_leaves(lvl[cur], w0, nleaf, chars, st);
    if (e != cudaSuccess) return cuda_status(e);
    h.resize(19 * w0 * nleaf);
    rc = device_to_host(h.data(), chars, h.size(), st);
    rc = check_device_error(rc);
    if (rc != BGPU_OK) return rc;
    size_t first = 0;
    while (first + 1 < h.size() && h[first] == '0') ++first;
    *first_out = first;
    g.last_launches = nl;
    return BGPU_OK;
}

static int to_decimal_locked(const uint32_t* digits, size_t n, bool neg, char* out, size_t out_cap,
                             size_t* out_len) {
    for (size_t i = 0; i < n; ++i)
        if (digits[i] >> 28) return BGPU_ERR_INVALID_ARG;
    n = strip32(digits, n);
    if (n == 0) {  // the reference prints zero as "0", without a sign
        *out_len = 1;
        if (out_cap < 1) return BGPU_ERR_OUT_CAPACITY;
        out[0] = '0';
        return BGPU_OK;
    }
    std::vector<char> h;
    size_t first = 0;
    const int rc = dec_chars(digits, nullptr, 0, n, digits[n - 1], &h, &first);
    if (rc != BGPU_OK) return rc;
    const size_t len = (h.size() - first) + (neg ? 1 : 0);
    *out_len = len;
    if (len > out_cap) return BGPU_ERR_OUT_CAPACITY;
    size_t o = 0;
    if (neg) out[o++] = '-';
    memcpy(out + o, h.data() + first, h.size() - first);
    return BGPU_OK;
}

// ---- BigFloat::print (src/bigint.cpp:972-1041) --------------------------------

// base^e (e >= 1) as a device value by the reference's fast_pow
// (include/bigint/bigint_base.h:60-69): multiply on a set bit, then square.
static int small_pow_val(uint32_t base, uint32_t e, DVal* out) {
    DVal b, r;
    int rc = upload_digits(kRsPowB0, std::vector<uint32_t>{base}, 0, false, &b);
    if (rc != BGPU_OK) return rc;
    bool have_r = false;
    int cb = 0, cr = 0;
    for (; e; e >>= 1) {
        if (e & 1) {
            if (!have_r) {  // res = 1 * base: a copy
                uint32_t* d = rslot(kRsPowR0 + cr, b.n, &rc);
                if (rc == BGPU_OK)
                    rc = cuda_status(cudaMemcpyAsync(d, b.d, b.n * 4, cudaMemcpyDeviceToDevice, g.stream));
                if (rc != BGPU_OK) return rc;
                r = b;
                r.d = d;
                r.slot = kRsPowR0 + cr;
                have_r = true;
            } else {
                DVal t;
                rc = int_product(r, b, kRsPowR0 + (cr ^ 1), &t);
                if (rc != BGPU_OK) return rc;
                cr ^= 1;
                r = t;
            }
        }
        if (e > 1) {  // the reference's last squaring does not change the result
            DVal t;
            rc = int_product(b, b, kRsPowB0 + (cb ^ 1), &t);
            if (rc != BGPU_OK) return rc;
            cb ^= 1;
            b = t;
        }
    }
    *out = r;
    return BGPU_OK;
}

// The reference's print of a BigFloat (digits, point position, sign) with
// dec_digits fraction digits (0: as many as the fraction's Digits hold):
//   int part = the digits above the point; frac = the digits below it;
//   F = BigInt(BigFloat(frac * 5^d, d - 28 pp), RoundHalfUp)   (= frac 10^d, rounded)
//   F == 10^d: F = 0, ++int part;
//   "-"? int "." F padded to d digits.
// The product, shift, rounding and comparison run as device steps; both
// parts are printed by the device decimal conversion.  Where the reference's
// rounding leaves no digits (2^-28 <= frac 10^d < 1/2; undefined behaviour),
// F is zero.
static int bigfloat_print_steps(const uint32_t* digits, size_t n, int64_t pp, bool neg, size_t dec_digits,
                                char* out, size_t out_cap, size_t* out_len) {
    if (n >= ((size_t)1 << 31)) return BGPU_ERR_CAPACITY;
    for (size_t i = 0; i < n; ++i)
        if (digits[i] >> 28) return BGPU_ERR_INVALID_ARG;
    if (n > 1 && digits[n - 1] == 0) return BGPU_ERR_INVALID_ARG;  // a leading zero digit
    const int64_t sn = (int64_t)n;
    // int part: digits [max(pp, 0), n) above -pp zero digits; {0} when pp >= n
    const size_t ilo = pp > 0 ? (size_t)pp : 0, ilow = pp < 0 ? (size_t)(-pp) : 0;
    size_t icount = pp < sn ? strip32(digits + ilo, n - ilo) : 0;
    // frac: digits [0, min(pp, n)); the default d counts them before leading zeros go
    const size_t fsize = pp > 0 ? (size_t)std::min(pp, sn) : 0;
    if (dec_digits == 0) dec_digits = (size_t)std::floor((double)(fsize * 28) * std::log10(2.0));
    if (dec_digits > ((size_t)1 << 28)) return BGPU_ERR_CAPACITY;
    const size_t fcount = strip32(digits, fsize);
    DVal F;  // zero
    bool carry = false;
    int rc = BGPU_OK;
    if (dec_digits && fcount) {
        DVal frac, K, X, S, T, one_pos, one_neg;
        rc = upload_int(kRsDivB, digits, fcount, false, &frac);
        if (rc == BGPU_OK) rc = small_pow_val(5, (uint32_t)dec_digits, &K);
        if (rc == BGPU_OK) rc = int_product(frac, K, kRsDivQB, &X);
        // BigFloat(X, -offset) with offset = 28 pp - d: X << (d - 28 pp), tail zeros removed
        if (rc == BGPU_OK) rc = shift_val(X, (int64_t)dec_digits - 28 * pp, kRsDivR, &S);
        if (rc != BGPU_OK) return rc;
        S.d += S.tz;
        S.n -= S.tz;
        S.pp -= (int64_t)S.tz;
        S.tz = 0;
        rc = upload_digits(kRsOne, std::vector<uint32_t>{1u}, 0, false, &one_pos);
        if (rc != BGPU_OK) return rc;
        one_neg = one_pos;
        one_neg.neg = true;
        rc = estimate_to_int(S, kRoundHalfUp, one_pos, one_neg, &F);
        // F == 10^d = 5^d << d ?
        if (rc == BGPU_OK && !F.zero()) rc = shift_val(K, (int64_t)dec_digits, kRsDivR2, &T);
        int c = 1;
        if (rc == BGPU_OK && !F.zero()) rc = cmp_abs(F, T, &c);
        if (rc != BGPU_OK) return rc;
        if (c == 0) {
            F = DVal{};
            carry = true;
        }
    }
    std::vector<char> ti, tf;
    size_t fi = 0, ff = 0;
    if (carry) {  // ++int part on the device
        DVal I, I1, one;
        rc = upload_digits(kRsOne, std::vector<uint32_t>{1u}, 0, false, &one);
        if (rc == BGPU_OK && icount) {
            uint32_t* d = rslot(kRsDivA, icount, &rc);
            if (rc == BGPU_OK) rc = host_to_device(d, digits + ilo, icount * 4, g.stream, nullptr);
            I = DVal{d, icount, -(int64_t)ilow, false, 0, digits[ilo + icount - 1], kRsDivA};
        }
        if (rc == BGPU_OK) rc = add_or_sub(I, one, false, kRsDivQ2, &I1);
        if (rc == BGPU_OK) rc = dec_chars(nullptr, I1.d, (size_t)(-I1.pp), I1.n, I1.top, &ti, &fi);
    } else {
        rc = dec_chars(digits + ilo, nullptr, icount ? ilow : 0, icount, icount ? digits[ilo + icount - 1] : 0,
                       &ti, &fi);
    }
    if (rc == BGPU_OK && dec_digits) {
        if (F.zero()) rc = dec_chars(nullptr, nullptr, 0, 0, 0, &tf, &ff);
        else rc = F.pp > 0 ? BGPU_ERR_CUDA : dec_chars(nullptr, F.d, (size_t)(-F.pp), F.n, F.top, &tf, &ff);
    }
    if (rc != BGPU_OK) return rc;
    const size_t li = ti.size() - fi, lf = dec_digits ? tf.size() - ff : 0;
    if (lf > dec_digits) return BGPU_ERR_CUDA;  // F < 10^d
    const size_t len = (neg ? 1 : 0) + li + 1 + dec_digits;
    *out_len = len;
    if (len > out_cap) return BGPU_ERR_OUT_CAPACITY;
    size_t o = 0;
    if (neg) out[o++] = '-';
    memcpy(out + o, ti.data() + fi, li);
    o += li;
    out[o++] = '.';
    memset(out + o, '0', dec_digits - lf);
    o += dec_digits - lf;
    if (lf) memcpy(out + o, tf.data() + ff, lf);
    return check_device_error(BGPU_OK);
}

int bgpu_bigfloat_to_decimal(const uint32_t* digits, size_t n, int64_t point_pos, int is_neg,
                             size_t dec_digits, char* out, size_t out_cap, size_t* out_len) {
    if (!digits || n == 0 || !out_len || (!out && out_cap)) return BGPU_ERR_INVALID_ARG;
    // 28 * point_pos and the shift d - 28 * point_pos stay far inside int64
    if (point_pos > BGPU_MAX_POINT_POS || point_pos < -BGPU_MAX_POINT_POS) return BGPU_ERR_CAPACITY;
    std::lock_guard<std::mutex> lk(g_mu);
    if (g.device < 0) return BGPU_ERR_NOT_INIT;
    cudaSetDevice(g.device);
    return with_device_status(
        bigfloat_print_steps(digits, n, point_pos, is_neg != 0, dec_digits, out, out_cap, out_len));
}

int bgpu_to_decimal(const uint32_t* digits, size_t n, int is_neg, char* out, size_t out_cap, size_t* out_len) {
    if (!digits || n == 0 || !out_len || (!out && out_cap)) return BGPU_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_mu);
    if (g.device < 0) return BGPU_ERR_NOT_INIT;
    cudaSetDevice(g.device);
    return with_device_status(to_decimal_locked(digits, n, is_neg != 0, out, out_cap, out_len));
}

int bgpu_from_decimal(const char* s, size_t len, uint32_t* out, size_t out_cap, size_t* out_len, int* is_neg) {
    if ((!s && len) || !out_len || !is_neg || (!out && out_cap)) return BGPU_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_mu);
    if (g.device < 0) return BGPU_ERR_NOT_INIT;
    cudaSetDevice(g.device);
    return with_device_status(from_decimal_locked(s, len, out, out_cap, out_len, is_neg));
}

int bgpu_batch_plan_create(const bgpu_product* products, size_t count, uint32_t flags,
                           bgpu_batch_plan* plan) {
    if (!plan || (!products && count)) return BGPU_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_mu);
    if (g.device < 0) return BGPU_ERR_NOT_INIT;
    cudaSetDevice(g.device);
    return batch_plan_create(products, count, flags, g.device, hooks_locked(), plan);
}

int bgpu_batch_plan_run(bgpu_batch_plan plan, void* stream) {
    if (!plan) return BGPU_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_mu);
    if (g.device < 0) return BGPU_ERR_NOT_INIT;
    cudaSetDevice(g.device);
    const int rc = batch_plan_run(plan, static_cast<cudaStream_t>(stream));
    if (rc == BGPU_OK) g.last_launches = batch_plan_launches(plan);
    return rc;
}

int bgpu_batch_plan_destroy(bgpu_batch_plan plan) {
    std::lock_guard<std::mutex> lk(g_mu);
    batch_plan_destroy(plan);
    return BGPU_OK;
}

uint32_t bgpu_batch_plan_launches(bgpu_batch_plan plan) { return batch_plan_launches(plan); }

int bgpu_mul_batch_device(const bgpu_product* products, size_t count, uint32_t flags, void* stream) {
    bgpu_batch_plan plan = nullptr;
    int rc = bgpu_batch_plan_create(products, count, flags, &plan);
    if (rc != BGPU_OK) return rc;
    rc = bgpu_batch_plan_run(plan, stream);
    if (rc == BGPU_OK) rc = bgpu_device_status(stream);
    bgpu_batch_plan_destroy(plan);
    return rc;
}

int bgpu_product_tree_device(const uint64_t* d_leaves, size_t n, uint64_t* d_out, size_t out_cap,
                             void* stream) {
    if (!d_leaves || !d_out || n == 0) return BGPU_ERR_INVALID_ARG;
    if (n > ((size_t)1 << 26)) return BGPU_ERR_CAPACITY;
    std::lock_guard<std::mutex> lk(g_mu);
    if (g.device < 0) return BGPU_ERR_NOT_INIT;
    cudaSetDevice(g.device);
    uint32_t nl = 0;
    int rc = product_tree_device(d_leaves, n, d_out, out_cap, hooks_locked(), &g.tree,
                                 static_cast<cudaStream_t>(stream), &nl);
    g.last_launches = nl;
    if (rc == BGPU_OK) rc = check_device_error(BGPU_OK);
    return rc;
}

int bgpu_product_tree_u64(const uint64_t* leaves, size_t n, uint64_t* out, size_t out_cap,
                          size_t* out_len) {
    if (!leaves || !out_len || n == 0 || (!out && out_cap)) return BGPU_ERR_INVALID_ARG;
    if (n > ((size_t)1 << 26)) return BGPU_ERR_CAPACITY;
    size_t width = 1;
    while (width < n) width <<= 1;
    std::lock_guard<std::mutex> lk(g_mu);
    if (g.device < 0) return BGPU_ERR_NOT_INIT;
    cudaSetDevice(g.device);
    int rc = ensure(&g.d_io, &g.io_bytes, align256(n * 8) + align256(width * 8));
    if (rc != BGPU_OK) return rc;
    uint64_t* dl = static_cast<uint64_t*>(g.d_io);
    uint64_t* dout = reinterpret_cast<uint64_t*>(static_cast<char*>(g.d_io) + align256(n * 8));
    rc = host_to_device(dl, leaves, n * 8, g.stream, nullptr);
    if (rc != BGPU_OK) return rc;
    uint32_t nl = 0;
    rc = product_tree_device(dl, n, dout, width, hooks_locked(), &g.tree, g.stream, &nl);
    g.last_launches = nl;
    if (rc != BGPU_OK) return rc;
    std::vector<uint64_t> tmp;
    uint64_t* dst = out;
    if (out_cap < width) {
        tmp.resize(width);
        dst = tmp.data();
    }
    rc = device_to_host(dst, dout, width * 8, g.stream);
    rc = check_device_error(rc);
    if (rc != BGPU_OK) return rc;
    const size_t len = strip64(dst, width);
    *out_len = len;
    if (dst != out) {
        if (len > out_cap) return BGPU_ERR_OUT_CAPACITY;
        memcpy(out, dst, len * 8);
    }
    return BGPU_OK;
}

int bgpu_set_block_limbs(uint64_t limbs) {
    if (limbs == 0) limbs = kHugeBlockLimbs;
    if (limbs < 64 || limbs > kHugeBlockLimbs || (limbs & (limbs - 1))) return BGPU_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_mu);
    g.huge_block = limbs;
    return BGPU_OK;
}

int bgpu_set_split(uint32_t log2_points, uint32_t log2_column) {
    std::lock_guard<std::mutex> lk(g_mu);
    return set_split((int)log2_points, (int)log2_column) == 0 ? BGPU_OK : BGPU_ERR_INVALID_ARG;
}

int bgpu_get_split(uint32_t log2_points) {
    if (log2_points < 5 || log2_points > kMaxLogN) return BGPU_ERR_INVALID_ARG;
    return choose_shape((int)log2_points).log_n2;
}

int bgpu_set_batch_split(uint32_t log2_points, uint32_t log2_column) {
    std::lock_guard<std::mutex> lk(g_mu);
    return set_batch_split((int)log2_points, (int)log2_column) == 0 ? BGPU_OK : BGPU_ERR_INVALID_ARG;
}

int bgpu_get_batch_split(uint32_t log2_points) {
    if (log2_points < 5 || log2_points > kMaxLogN) return BGPU_ERR_INVALID_ARG;
    return choose_shape_batch((int)log2_points).log_n2;
}

int bgpu_set_tuning(uint32_t key, uint64_t value) {
    std::lock_guard<std::mutex> lk(g_mu);
    Tuning& t = g_tuning;
    switch (key) {
        case BGPU_TUNE_SCHOOLBOOK_MAX_LIMBS:
            if (value > kSchoolbookMaxLimbs) return BGPU_ERR_INVALID_ARG;
            t.schoolbook_max_limbs = (uint32_t)value;
            return BGPU_OK;
        case BGPU_TUNE_BATCH_SCHOOLBOOK_MAX_LIMBS:
            if (value > kSchoolbookMaxLimbs) return BGPU_ERR_INVALID_ARG;
            t.batch_schoolbook_max_limbs = (uint32_t)value;
            return BGPU_OK;
        case BGPU_TUNE_FFT_MIN_LIMBS: t.fft_min_limbs = value; return BGPU_OK;
        case BGPU_TUNE_FFT_MAX_LIMBS: t.fft_max_limbs = value; return BGPU_OK;
        case BGPU_TUNE_KARATSUBA_MAX_LIMBS:
            if (value > 2 * kKaratsubaMaxLimbs) return BGPU_ERR_INVALID_ARG;
            t.karatsuba_max_limbs = (uint32_t)value;
            return BGPU_OK;
        case BGPU_TUNE_BATCH_KARATSUBA_MAX_LIMBS:
            if (value > 2 * kKaratsubaMaxLimbs) return BGPU_ERR_INVALID_ARG;
            t.batch_karatsuba_max_limbs = (uint32_t)value;
            return BGPU_OK;
        default: return BGPU_ERR_INVALID_ARG;
    }
}

int bgpu_get_tuning(uint32_t key, uint64_t* value) {
    if (!value) return BGPU_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_mu);
    const Tuning& t = g_tuning;
    switch (key) {
        case BGPU_TUNE_SCHOOLBOOK_MAX_LIMBS: *value = t.schoolbook_max_limbs; return BGPU_OK;
        case BGPU_TUNE_BATCH_SCHOOLBOOK_MAX_LIMBS: *value = t.batch_schoolbook_max_limbs; return BGPU_OK;
        case BGPU_TUNE_FFT_MIN_LIMBS: *value = t.fft_min_limbs; return BGPU_OK;
        case BGPU_TUNE_FFT_MAX_LIMBS: *value = t.fft_max_limbs; return BGPU_OK;
        case BGPU_TUNE_KARATSUBA_MAX_LIMBS: *value = t.karatsuba_max_limbs; return BGPU_OK;
        case BGPU_TUNE_BATCH_KARATSUBA_MAX_LIMBS: *value = t.batch_karatsuba_max_limbs; return BGPU_OK;
        default: return BGPU_ERR_INVALID_ARG;
    }
}

int bgpu_load_tuning(const char* path) {
    if (!path) return BGPU_ERR_INVALID_ARG;
    FILE* f = fopen(path, "r");
    if (!f) return BGPU_ERR_INVALID_ARG;
    // Parse everything first, apply only a fully valid table.
    struct Split { unsigned ln, l2; bool batch; };
    std::vector<Split> splits;
    std::vector<std::pair<uint32_t, unsigned long long>> vals;
    char line[256];
    int rc = BGPU_OK;
    while (rc == BGPU_OK && fgets(line, sizeof line, f)) {
        char key[64];
        unsigned long long a = 0, b = 0;
        const char* p = line;
        while (*p == ' ' || *p == '\t') ++p;
        if (*p == '#' || *p == '\n' || *p == '\0') continue;
        const int n = sscanf(p, "%63s %llu %llu", key, &a, &b);
        if (n >= 3 && strcmp(key, "split") == 0) {
            splits.push_back({(unsigned)a, (unsigned)b, false});
        } else if (n >= 3 && strcmp(key, "batch_split") == 0) {
            splits.push_back({(unsigned)a, (unsigned)b, true});
        } else if (n == 2 && strcmp(key, "schoolbook_max_limbs") == 0) {
            vals.push_back({BGPU_TUNE_SCHOOLBOOK_MAX_LIMBS, a});
        } else if (n == 2 && strcmp(key, "batch_schoolbook_max_limbs") == 0) {
            vals.push_back({BGPU_TUNE_BATCH_SCHOOLBOOK_MAX_LIMBS, a});
        } else if (n == 2 && strcmp(key, "fft_min_limbs") == 0) {
            vals.push_back({BGPU_TUNE_FFT_MIN_LIMBS, a});
        } else if (n == 2 && strcmp(key, "fft_max_limbs") == 0) {
            vals.push_back({BGPU_TUNE_FFT_MAX_LIMBS, a});
        } else if (n == 2 && strcmp(key, "karatsuba_max_limbs") == 0) {
            vals.push_back({BGPU_TUNE_KARATSUBA_MAX_LIMBS, a});
        } else if (n == 2 && strcmp(key, "batch_karatsuba_max_limbs") == 0) {
            vals.push_back({BGPU_TUNE_BATCH_KARATSUBA_MAX_LIMBS, a});
        } else {
            rc = BGPU_ERR_INVALID_ARG;
        }
    }
    fclose(f);
    if (rc != BGPU_OK) return rc;
    for (const Split& sp : splits) {
        const int l1 = (int)sp.ln - (int)sp.l2;
        if (sp.ln < 5 || sp.ln > (unsigned)kMaxLogN || sp.l2 < 2 || sp.l2 > 11 || l1 < 3 || l1 > 15)
            return BGPU_ERR_INVALID_ARG;
    }
    for (auto& kv : vals) {
        if ((kv.first == BGPU_TUNE_SCHOOLBOOK_MAX_LIMBS || kv.first == BGPU_TUNE_BATCH_SCHOOLBOOK_MAX_LIMBS) &&
            kv.second > kSchoolbookMaxLimbs)
            return BGPU_ERR_INVALID_ARG;
        if ((kv.first == BGPU_TUNE_KARATSUBA_MAX_LIMBS || kv.first == BGPU_TUNE_BATCH_KARATSUBA_MAX_LIMBS) &&
            kv.second > 2 * kKaratsubaMaxLimbs)
            return BGPU_ERR_INVALID_ARG;
    }
    for (const Split& sp : splits) {
        if (sp.batch) bgpu_set_batch_split(sp.ln, sp.l2);
        else bgpu_set_split(sp.ln, sp.l2);
    }
    for (auto& kv : vals) bgpu_set_tuning(kv.first, kv.second);
    return BGPU_OK;
}

int bgpu_set_kernel_timing(int on) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (g.device < 0) return BGPU_ERR_NOT_INIT;
    cudaSetDevice(g.device);
    if (on && g.kev.empty()) {
        g.kev.resize((size_t)kTimingRing * (kNttLaunches + 1));
        for (auto& e : g.kev) {
            if (cudaEventCreate(&e) != cudaSuccess) {
                for (auto x : g.kev)
                    if (x) cudaEventDestroy(x);
                g.kev.clear();
                return BGPU_ERR_CUDA;
            }
        }
    }
    g.kernel_timing = on != 0;
    if (on) g.kev_count = 0;
    return BGPU_OK;
}

int bgpu_kernel_times(const char** names, float* mean_ms, int cap, uint32_t* nproducts) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (g.device < 0) return BGPU_ERR_NOT_INIT;
    if (nproducts) *nproducts = 0;
    if (g.kev_count == 0 || g.kev.empty()) return 0;
    cudaSetDevice(g.device);
    const uint64_t n = g.kev_count < kTimingRing ? g.kev_count : kTimingRing;
    const size_t last = ((g.kev_count - 1) % kTimingRing) * (kNttLaunches + 1) + kNttLaunches;
    if (cudaEventSynchronize(g.kev[last]) != cudaSuccess) return BGPU_ERR_CUDA;
    int k = 0;
    for (; k < kNttLaunches && k < cap; ++k) {
        double sum = 0;
        for (uint64_t i = 0; i < n; ++i) {
            float t = 0;
            const cudaEvent_t* ev = g.kev.data() + i * (kNttLaunches + 1);
            if (cudaEventElapsedTime(&t, ev[k], ev[k + 1]) != cudaSuccess) return BGPU_ERR_CUDA;
            sum += t;
        }
        if (names) names[k] = kNttKernelNames[k];
        if (mean_ms) mean_ms[k] = (float)(sum / (double)n);
    }
    if (nproducts) *nproducts = (uint32_t)n;
    return k;
}

}  // extern "C"
