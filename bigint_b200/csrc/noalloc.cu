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
//   * the static arrays (about 3.8 MB of scratch plus 0.35 MB of tables) are
//     held by every GPU that loads this library until the process exits;
//   * every call shares the one scratch array, which keeps the last call's
//     contents; the carry-scan ticket, flags and error word are cleared on the
//     caller's stream at the start of each call, the rest is fully rewritten.
//     Calls within one process are serialized per device: a host mutex is
//     held until the call's work has finished, so their work cannot overlap
//     on the GPU (work that did overlap would race on the array).  Each
//     process has its own copy of the array.
//   * the first call on each device performs the set-up (table upload and
//     cudaGetSymbolAddress, synchronous); make that first call before any
//     stream capture.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/bigint_b200.h"
#include "engine.h"
#include "tables.h"

namespace bgpu {
namespace {

constexpr int kNaLogN = 17;                   // largest transform of this entry point
constexpr size_t kNaPoints = (size_t)1 << kNaLogN;
constexpr int kNaStageLog = 10;               // stage tables cover pair distances < 2^10

constexpr size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kOffY = 0;
constexpr size_t kOffChunks = kOffY + al256(2 * (size_t)kNumPrimes * kNaPoints * 4);
constexpr size_t kOffSpill = kOffChunks + al256(kNaPoints / 2 * 8);
constexpr size_t kOffFlags = kOffSpill + al256(kNaPoints / 8 * 8);
constexpr size_t kFlagWords = (kNaPoints / 8 + kCarryChunksPerBlock) / kCarryChunksPerBlock;  // carry-scan blocks
constexpr size_t kOffTicket = kOffFlags + al256(kFlagWords * 8);
constexpr size_t kOffErr = kOffTicket + 256;
constexpr size_t kScratchBytes = kOffErr + 256;

constexpr int kNaSet = 0;  // every product here fits the lazy prime set

}  // namespace

// The scratch array and the twiddle tables of this entry point.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];
static __device__ __align__(256) uint2 g_noalloc_tables[table_entries(kNaSet, kNaStageLog)];

namespace {

// Host-side copy used only to build the tables (static, no heap).
uint2 h_tables[table_entries(kNaSet, kNaStageLog)];

struct DeviceSetup {
    bool ready = false;
    NttConsts consts{};
    unsigned char* scratch = nullptr;  // device address of g_noalloc_scratch
};

constexpr int kMaxDevices = 64;
DeviceSetup g_setup[kMaxDevices];
std::mutex g_na_mu[kMaxDevices];  // one per device: its set-up and its use of the scratch

// Once per device, with that device current: upload the tables and take the
// device addresses of the static arrays.  In host code the array names are
// host-side stand-ins, so only the addresses from cudaGetSymbolAddress are
// ever handed to a kernel.
int setup_device(int dev, DeviceSetup* s) {
    build_tables(kNaSet, kNaStageLog, h_tables);
    if (cudaMemcpyToSymbol(g_noalloc_tables, h_tables, sizeof(h_tables)) != cudaSuccess)
        return BGPU_ERR_CUDA;
    void* scratch = nullptr;
    void* tables = nullptr;
    if (cudaGetSymbolAddress(&scratch, g_noalloc_scratch) != cudaSuccess) return BGPU_ERR_CUDA;
    if (cudaGetSymbolAddress(&tables, g_noalloc_tables) != cudaSuccess) return BGPU_ERR_CUDA;
    s->scratch = static_cast<unsigned char*>(scratch);
    s->consts = make_consts(kNaSet, kNaStageLog, static_cast<const uint2*>(tables));
    if (upload_consts(kSlotNoAlloc + kNaSet, s->consts) != cudaSuccess) return BGPU_ERR_CUDA;
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
    std::lock_guard<std::mutex> lk(g_na_mu[dev]);
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
    // The static stage tables cover rows and columns up to 2^kNaStageLog
    // points, which the built-in split keeps to for every length here; a
    // tuned split (bgpu_set_split) may not, so it is not used.
    const TransformShape shape = builtin_shape(log_n);
    if (shape.log_n1 > kNaStageLog || shape.log_n2 > kNaStageLog) return BGPU_ERR_CAPACITY;
    cudaError_t e = launch_ntt_product(kSlotNoAlloc + kNaSet, s.consts, oa, ob, square, log_n, ps,
                                       d_out, kFmtLimb64, na + nb, cl, st, nullptr, &shape);
    if (e != cudaSuccess) {
        // Kernels queued before the failing launch still write the scratch:
        // let them finish before the lock goes, so the next call's clearing
        // of the carry-scan state cannot race them.
        cudaStreamSynchronize(st);
        return e == cudaErrorMemoryAllocation ? BGPU_ERR_OOM : BGPU_ERR_CUDA;
    }
    // Synchronous completion: wait for the product and report a bounded
    // device-side wait that gave up (the error word is part of the scratch).
    uint32_t err = 0;
    e = cudaMemcpyAsync(&err, ps.err, sizeof(err), cudaMemcpyDeviceToHost, st);
    const cudaError_t es = cudaStreamSynchronize(st);
    if (e != cudaSuccess || es != cudaSuccess) return BGPU_ERR_CUDA;
    return err ? BGPU_ERR_DEVICE_TIMEOUT : BGPU_OK;
}
