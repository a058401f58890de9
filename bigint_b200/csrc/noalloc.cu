// No-allocation entry point: the NTT product with its scratch in static
// device memory.
//
// Some callers cannot allocate device memory at the point they multiply:
// code that runs under a caller-owned memory budget or pool that must not
// grow, host threads that may not call cudaMalloc (it can synchronize the
// device), or a process that pre-plans every byte it uses on the GPU.
// bgpu_mul_u64_device_noalloc serves them: it runs the same four NTT kernels
// as bgpu_mul_u64_device, but every scratch buffer (residue planes, chunk
// sums, spills, carry-scan flags, ticket, error word) lives in the file-scope
// array g_noalloc_scratch below and the twiddle tables in file-scope arrays
// too.  Nothing is allocated: no cudaMalloc / cudaFree / allocating library
// routine, and no host heap (the tables are built in static host arrays).
//
// Limits and sharing:
//   * the product must satisfy na + nb <= BGPU_NOALLOC_MAX_LIMBS (65536 u64
//     limbs, i.e. at most 2^17 transform points); larger products are
//     rejected with BGPU_ERR_CAPACITY before anything is launched;
//   * the static arrays (about 3.8 MB of scratch plus 0.8 MB of tables) are
//     held by every GPU that loads this library until the process exits;
//   * every call shares the one scratch array, which keeps the last call's
//     contents; the carry-scan ticket, flags and error word are cleared on the
//     caller's stream at the start of each call, the rest is fully rewritten.
//     Calls whose work overlaps on the GPU (two streams, two host threads)
//     race on the array and must be serialized by the caller.
//   * the first call on each device performs the set-up (table upload and
//     cudaGetSymbolAddress, synchronous); make that first call before any
//     stream capture.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/bigint_b200.h"
#include "engine.h"

namespace bgpu {
namespace {

constexpr int kNaLogN = 17;                   // largest transform of this entry point
constexpr size_t kNaPoints = (size_t)1 << kNaLogN;
constexpr int kNaStageLog = 10;               // stage tables cover pair distances < 2^10
constexpr size_t kNaSplit = (size_t)1 << kTwSplit;

constexpr size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kOffY = 0;
constexpr size_t kOffChunks = kOffY + al256(2 * (size_t)kNumPrimes * kNaPoints * 4);
constexpr size_t kOffSpill = kOffChunks + al256(kNaPoints / 2 * 8);
constexpr size_t kOffFlags = kOffSpill + al256(kNaPoints / 8 * 8);
constexpr size_t kFlagWords = (kNaPoints / 8 + 1 + 255) / 256;  // carry-scan blocks
constexpr size_t kOffTicket = kOffFlags + al256(kFlagWords * 8);
constexpr size_t kOffErr = kOffTicket + 256;
constexpr size_t kScratchBytes = kOffErr + 256;

constexpr uint32_t kNaPrimes[kNumPrimes] = {469762049u, 1811939329u, 2013265921u};
constexpr uint32_t kNaGens[kNumPrimes] = {3u, 13u, 31u};

}  // namespace

// The scratch array and the twiddle tables of this entry point.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];
static __device__ __align__(256) uint2 g_noalloc_stage[kNumPrimes][2][(size_t)1 << kNaStageLog];
static __device__ __align__(256) uint2 g_noalloc_split[kNumPrimes][2][2][kNaSplit];

namespace {

// Host-side copies used only to build the tables (static, no heap).
uint2 h_stage[kNumPrimes][2][(size_t)1 << kNaStageLog];
uint2 h_split[kNumPrimes][2][2][kNaSplit];

struct DeviceSetup {
    bool ready = false;
    NttConsts consts{};
    unsigned char* scratch = nullptr;  // device address of g_noalloc_scratch
};

constexpr int kMaxDevices = 64;
DeviceSetup g_setup[kMaxDevices];
std::mutex g_na_mu;

uint64_t na_pow(uint64_t b, uint64_t e, uint64_t p) {
    uint64_t r = 1;
    b %= p;
    while (e) {
        if (e & 1) r = r * b % p;
        b = b * b % p;
        e >>= 1;
    }
    return r;
}

uint32_t na_inv32(uint32_t p) {
    uint32_t x = 1;
    for (int i = 0; i < 5; ++i) x *= 2u - p * x;
    return x;
}

uint2 na_mont(uint64_t v, uint32_t p) {
    const uint32_t w = (uint32_t)(((v % p) << 32) % p);
    return make_uint2(w, w * na_inv32(p));
}

void build_host_tables() {
    for (int q = 0; q < kNumPrimes; ++q) {
        const uint32_t p = kNaPrimes[q];
        for (int dir = 0; dir < 2; ++dir) {
            uint2* st = h_stage[q][dir];
            st[0] = na_mont(1, p);
            for (size_t h = 1; h < ((size_t)1 << kNaStageLog); h <<= 1) {
                uint64_t root = na_pow(kNaGens[q], (p - 1) / (2 * h), p);
                if (dir) root = na_pow(root, p - 2, p);
                uint64_t v = 1;
                for (size_t m = 0; m < h; ++m) {
                    st[h + m] = na_mont(v, p);
                    v = v * root % p;
                }
            }
            uint64_t r26 = na_pow(kNaGens[q], (p - 1) >> kMaxLogN, p);
            if (dir) r26 = na_pow(r26, p - 2, p);
            const uint64_t step_hi = na_pow(r26, kNaSplit, p);
            uint64_t vh = 1, vl = 1;
            for (size_t i = 0; i < kNaSplit; ++i) {
                h_split[q][dir][0][i] = na_mont(vh, p);
                h_split[q][dir][1][i] = na_mont(vl, p);
                vh = vh * step_hi % p;
                vl = vl * r26 % p;
            }
        }
    }
}

// Once per device, with that device current: upload the tables and take the
// device addresses of the static arrays.  In host code the array names are
// host-side stand-ins, so only the addresses from cudaGetSymbolAddress are
// ever handed to a kernel.
int setup_device(int dev, DeviceSetup* s) {
    build_host_tables();
    if (cudaMemcpyToSymbol(g_noalloc_stage, h_stage, sizeof(h_stage)) != cudaSuccess)
        return BGPU_ERR_CUDA;
    if (cudaMemcpyToSymbol(g_noalloc_split, h_split, sizeof(h_split)) != cudaSuccess)
        return BGPU_ERR_CUDA;
    void* scratch = nullptr;
    void* stage = nullptr;
    void* split = nullptr;
    if (cudaGetSymbolAddress(&scratch, g_noalloc_scratch) != cudaSuccess) return BGPU_ERR_CUDA;
    if (cudaGetSymbolAddress(&stage, g_noalloc_stage) != cudaSuccess) return BGPU_ERR_CUDA;
    if (cudaGetSymbolAddress(&split, g_noalloc_split) != cudaSuccess) return BGPU_ERR_CUDA;
    s->scratch = static_cast<unsigned char*>(scratch);
    const uint2* st = static_cast<const uint2*>(stage);
    const uint2* sp = static_cast<const uint2*>(split);
    NttConsts& c = s->consts;
    for (int q = 0; q < kNumPrimes; ++q) {
        c.pr[q].p = kNaPrimes[q];
        c.pr[q].pinv = na_inv32(kNaPrimes[q]);
        const uint2 one = na_mont(1, kNaPrimes[q]);
        c.one_w[q] = one.x;
        c.one_wp[q] = one.y;
        for (int dir = 0; dir < 2; ++dir) {
            c.stage[q][dir] = st + ((size_t)q * 2 + dir) * ((size_t)1 << kNaStageLog);
            c.th[q][dir] = sp + (((size_t)q * 2 + dir) * 2 + 0) * kNaSplit;
            c.tl[q][dir] = sp + (((size_t)q * 2 + dir) * 2 + 1) * kNaSplit;
        }
    }
    const uint32_t p0 = kNaPrimes[0], p1 = kNaPrimes[1], p2 = kNaPrimes[2];
    const uint2 k1 = na_mont(na_pow(p0, p1 - 2, p1), p1);
    const uint2 k2 = na_mont(p0 % p2, p2);
    const uint2 k3 = na_mont(na_pow((uint64_t)p0 * p1 % p2, p2 - 2, p2), p2);
    c.k1 = k1.x, c.k1p = k1.y;
    c.k2 = k2.x, c.k2p = k2.y;
    c.k3 = k3.x, c.k3p = k3.y;
    c.m01 = (uint64_t)p0 * p1;
    if (cudaMemset(s->scratch + kOffErr, 0, sizeof(uint32_t)) != cudaSuccess) return BGPU_ERR_CUDA;
    (void)dev;
    s->ready = true;
    return BGPU_OK;
}

}  // namespace
}  // namespace bgpu

using namespace bgpu;

extern "C" int bgpu_mul_u64_device_noalloc(const uint64_t* d_a, size_t na, const uint64_t* d_b,
                                           size_t nb, uint64_t* d_out, void* stream) {
    if (!d_a || !d_b || !d_out || na == 0 || nb == 0) return BGPU_ERR_INVALID_ARG;
    if (na + nb > BGPU_NOALLOC_MAX_LIMBS) return BGPU_ERR_CAPACITY;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return BGPU_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lk(g_na_mu);
    DeviceSetup& s = g_setup[dev];
    if (!s.ready) {
        const int rc = setup_device(dev, &s);
        if (rc != BGPU_OK) return rc;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool square = (d_a == d_b && na == nb);
    const uint64_t total32 = 2 * (uint64_t)(na + nb);
    int log_n = 0;
    while (((uint64_t)1 << log_n) < total32 - 1) ++log_n;
    if (log_n < 5) log_n = 5;
    if (log_n > kNaLogN) return BGPU_ERR_CAPACITY;

    ProductScratch ps{};
    ps.y = reinterpret_cast<uint32_t*>(s.scratch + kOffY);
    ps.chunks = reinterpret_cast<uint64_t*>(s.scratch + kOffChunks);
    ps.spill = reinterpret_cast<uint64_t*>(s.scratch + kOffSpill);
    ps.flags = reinterpret_cast<uint64_t*>(s.scratch + kOffFlags);
    ps.ticket = reinterpret_cast<unsigned long long*>(s.scratch + kOffTicket);
    ps.err = reinterpret_cast<uint32_t*>(s.scratch + kOffErr);
    // The previous call's carry-scan state must not leak into this one: the
    // ticket restarts at 0 and all flag words are cleared (epoch 0 is never
    // a valid epoch, so the scan uses epoch 1 every call).
    if (cudaMemsetAsync(ps.flags, 0, kFlagWords * 8, st) != cudaSuccess) return BGPU_ERR_CUDA;
    if (cudaMemsetAsync(ps.ticket, 0, 8, st) != cudaSuccess) return BGPU_ERR_CUDA;
    if (cudaMemsetAsync(ps.err, 0, 4, st) != cudaSuccess) return BGPU_ERR_CUDA;
    CarryLaunch cl;
    cl.ticket_base = 0;
    cl.epoch = 1;
    OperandDesc oa{d_a, (uint32_t)na, (uint32_t)(2 * na), kFmtLimb64};
    OperandDesc ob{d_b, (uint32_t)nb, (uint32_t)(2 * nb), kFmtLimb64};
    cudaError_t e = launch_ntt_product(s.consts, oa, ob, square, log_n, ps, d_out, kFmtLimb64,
                                       na + nb, cl, st, nullptr);
    if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? BGPU_ERR_OOM : BGPU_ERR_CUDA;
    // Synchronous completion: wait for the product and report a bounded
    // device-side wait that gave up (the error word is part of the scratch).
    uint32_t err = 0;
    e = cudaMemcpyAsync(&err, ps.err, sizeof(err), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return BGPU_ERR_CUDA;
    return err ? BGPU_ERR_DEVICE_TIMEOUT : BGPU_OK;
}
