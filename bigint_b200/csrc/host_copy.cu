// Host <-> device copies of the host API.
//
// The reference hands its operands over in ordinary (pageable) heap memory:
// std::vector<uint64_t> limbs and Digits.  A pageable cudaMemcpyAsync runs
// at a fraction of the copy engines' rate because the driver stages it
// through its own small page-locked buffer with one host thread.  This file
// stages it instead through a ring of engine-owned page-locked slots, splits
// the host-side memcpy of every slot over a pool of worker threads and
// overlaps it with the DMA of the previous slot.  Page-locked caller memory
// (cudaHostAlloc / cudaHostRegister / torch pin_memory) and small copies go
// straight to cudaMemcpyAsync.
//
// The 28-bit check of the reference's Digits (every digit < 2^28,
// include/bigint/mul.h:223) is folded into the same pass over the caller's
// memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/bigint_b200.h"
#include "engine.h"

namespace bgpu {
namespace {

constexpr size_t kPiece = 256 << 10;      // bytes one worker copies at a time
constexpr size_t kSlot = 4 << 20;         // bytes of one page-locked slot
constexpr int kSlots = 4;                 // slots in the ring
constexpr size_t kDirectMax = 256 << 10;  // pageable copies up to this go to the driver
constexpr unsigned kMaxWorkers = 16;
constexpr auto kSpin = std::chrono::microseconds(200);  // idle workers poll this long before sleeping

inline void cpu_relax() {
#if defined(__x86_64__) || defined(__i386__)
    __builtin_ia32_pause();
#else
    std::this_thread::yield();
#endif
}

// Fixed pool of host threads running index-parallel jobs.  The calling thread
// takes part, so a job finishes even with no worker running (after fork()).
// The job counter carries the job's generation in its high half: a worker
// that picked up an older job's parameters never claims an index of a newer
// one.  One call of the host API runs several jobs back to back (operand
// copies, then the result's), so an idle worker polls for the next job for a
// short while before it sleeps on the condition variable.
class Pool {
  public:
    ~Pool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_.store(true);
        }
        cv_.notify_all();
        for (auto& t : threads_) t.join();
    }

    void run(uint32_t n, void (*fn)(void*, uint32_t), void* ctx) {
        if (n == 0) return;
        start();
        uint32_t gen;
        {
            std::lock_guard<std::mutex> lk(mu_);
            gen = ++gen_;
            fn_ = fn;
            ctx_ = ctx;
            n_ = n;
            done_.store(0, std::memory_order_relaxed);
            next_.store((uint64_t)gen << 32, std::memory_order_release);
            pub_.store(gen, std::memory_order_release);
        }
        if (n > 1) cv_.notify_all();
        work(gen, n, fn, ctx);
        while (done_.load(std::memory_order_acquire) < n) std::this_thread::yield();
    }

  private:
    void start() {
        if (started_) return;
        started_ = true;
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const unsigned nw = std::min(hw, kMaxWorkers) - 1;
        for (unsigned i = 0; i < nw; ++i) threads_.emplace_back([this] { loop(); });
    }

    void work(uint32_t gen, uint32_t n, void (*fn)(void*, uint32_t), void* ctx) {
        for (;;) {
            uint64_t v = next_.load(std::memory_order_acquire);
            if ((uint32_t)(v >> 32) != gen || (uint32_t)v >= n) return;
            if (!next_.compare_exchange_weak(v, v + 1, std::memory_order_acq_rel)) continue;
            fn(ctx, (uint32_t)v);
            done_.fetch_add(1, std::memory_order_release);
        }
    }

    void loop() {
        uint32_t seen = 0;
        for (;;) {
            uint32_t gen, n;
            void (*fn)(void*, uint32_t);
            void* ctx;
            const auto t0 = std::chrono::steady_clock::now();
            for (uint32_t i = 1; pub_.load(std::memory_order_acquire) == seen && !stop_.load(); ++i) {
                cpu_relax();
                if ((i & 255) == 0 && std::chrono::steady_clock::now() - t0 > kSpin) break;
            }
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_.load() || gen_ != seen; });
                if (stop_.load()) return;
                seen = gen = gen_;
                fn = fn_;
                ctx = ctx_;
                n = n_;
            }
            work(gen, n, fn, ctx);
        }
    }

    std::vector<std::thread> threads_;
    bool started_ = false;
    std::mutex mu_;
    std::condition_variable cv_;
    std::atomic<bool> stop_{false};
    uint32_t gen_ = 0;                 // written under mu_
    std::atomic<uint32_t> pub_{0};     // gen_, for the polling workers
    void (*fn_)(void*, uint32_t) = nullptr;
    void* ctx_ = nullptr;
    uint32_t n_ = 0;
    std::atomic<uint64_t> next_{0};
    std::atomic<uint32_t> done_{0};
};

Pool g_pool;

struct Ring {
    char* host = nullptr;  // kSlots * kSlot page-locked bytes
    cudaEvent_t ev[kSlots] = {};
    bool busy[kSlots] = {};
    int next = 0;
};

Ring g_ring;

int status(cudaError_t e) {
    if (e == cudaSuccess) return BGPU_OK;
    if (e == cudaErrorMemoryAllocation) return BGPU_ERR_OOM;
    return BGPU_ERR_CUDA;
}

int ring_ready() {
    if (g_ring.host) return BGPU_OK;
    cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&g_ring.host), kSlots * kSlot, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        cudaGetLastError();
        g_ring.host = nullptr;
        return status(e);
    }
    for (int k = 0; k < kSlots && e == cudaSuccess; ++k)
        e = cudaEventCreateWithFlags(&g_ring.ev[k], cudaEventDisableTiming);
    if (e != cudaSuccess) {
        release_host_staging();
        return status(e);
    }
    return BGPU_OK;
}

// Claims the next slot once the copy that used it last has finished.
int claim(int* slot) {
    const int k = g_ring.next;
    g_ring.next = (k + 1) % kSlots;
    if (g_ring.busy[k]) {
        cudaError_t e = cudaEventSynchronize(g_ring.ev[k]);
        if (e != cudaSuccess) return status(e);
        g_ring.busy[k] = false;
    }
    *slot = k;
    return BGPU_OK;
}

bool page_locked(const void* p) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

struct CopyJob {
    char* dst;
    const char* src;
    size_t bytes;
    uint32_t* hi28;  // nullptr, or one OR of (digit >> 28) per piece
};

void copy_piece(void* c, uint32_t i) {
    const CopyJob& j = *static_cast<const CopyJob*>(c);
    const size_t off = (size_t)i * kPiece, len = std::min(kPiece, j.bytes - off);
    if (!j.hi28) {
        memcpy(j.dst + off, j.src + off, len);
        return;
    }
    // Digits: copy and check together (offsets and lengths are multiples of 4)
    const uint32_t* s = reinterpret_cast<const uint32_t*>(j.src + off);
    uint32_t* d = reinterpret_cast<uint32_t*>(j.dst + off);
    uint32_t acc = 0;
    for (size_t w = 0; w < len / 4; ++w) {
        const uint32_t x = s[w];
        d[w] = x;
        acc |= x;
    }
    j.hi28[i] = acc >> 28;
}

void check_piece(void* c, uint32_t i) {
    const CopyJob& j = *static_cast<const CopyJob*>(c);
    const size_t off = (size_t)i * kPiece, len = std::min(kPiece, j.bytes - off);
    const uint32_t* s = reinterpret_cast<const uint32_t*>(j.src + off);
    uint32_t acc = 0;
    for (size_t w = 0; w < len / 4; ++w) acc |= s[w];
    j.hi28[i] = acc >> 28;
}

// Parallel copy (dst != nullptr) and/or check of `bytes` host bytes; returns
// the OR of the pieces' checks (0 when check is false).
uint32_t host_copy(char* dst, const char* src, size_t bytes, bool check) {
    const uint32_t pieces = (uint32_t)((bytes + kPiece - 1) / kPiece);
    uint32_t hi[kSlot / kPiece + 1];
    std::vector<uint32_t> big;
    uint32_t* h = nullptr;
    if (check) {
        if (pieces <= sizeof(hi) / sizeof(hi[0])) {
            h = hi;
        } else {
            big.resize(pieces);
            h = big.data();
        }
    }
    CopyJob j{dst, src, bytes, h};
    g_pool.run(pieces, dst ? copy_piece : check_piece, &j);
    uint32_t acc = 0;
    for (uint32_t i = 0; check && i < pieces; ++i) acc |= h[i];
    return acc;
}

}  // namespace

int host_to_device(void* dst, const void* src, size_t bytes, cudaStream_t st, bool* digits_ok) {
    if (digits_ok) *digits_ok = true;
    if (bytes == 0) return BGPU_OK;
    if (bytes <= kDirectMax || page_locked(src)) {
        if (digits_ok) *digits_ok = host_copy(nullptr, static_cast<const char*>(src), bytes, true) == 0;
        return status(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
    }
    int rc = ring_ready();
    if (rc != BGPU_OK) return rc;
    uint32_t hi = 0;
    for (size_t off = 0; off < bytes; off += kSlot) {
        const size_t len = std::min(kSlot, bytes - off);
        int k;
        rc = claim(&k);
        if (rc != BGPU_OK) return rc;
        char* slot = g_ring.host + (size_t)k * kSlot;
        hi |= host_copy(slot, static_cast<const char*>(src) + off, len, digits_ok != nullptr);
        cudaError_t e = cudaMemcpyAsync(static_cast<char*>(dst) + off, slot, len, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaEventRecord(g_ring.ev[k], st);
        if (e != cudaSuccess) return status(e);
        g_ring.busy[k] = true;
    }
    if (digits_ok) *digits_ok = hi == 0;
    return BGPU_OK;
}

int device_to_host(void* dst, const void* src, size_t bytes, cudaStream_t st) {
    if (bytes == 0) return BGPU_OK;
    if (bytes <= kDirectMax || page_locked(dst)) {
        cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        return status(e);
    }
    int rc = ring_ready();
    if (rc != BGPU_OK) return rc;
    const size_t chunks = (bytes + kSlot - 1) / kSlot;
    int slot_of[kSlots];
    auto issue = [&](size_t c) -> int {
        int k;
        int r = claim(&k);
        if (r != BGPU_OK) return r;
        const size_t off = c * kSlot, len = std::min(kSlot, bytes - off);
        cudaError_t e = cudaMemcpyAsync(g_ring.host + (size_t)k * kSlot, static_cast<const char*>(src) + off,
                                        len, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaEventRecord(g_ring.ev[k], st);
        if (e != cudaSuccess) return status(e);
        g_ring.busy[k] = true;
        slot_of[c % kSlots] = k;
        return BGPU_OK;
    };
    for (size_t c = 0; c < chunks && c < (size_t)kSlots; ++c) {
        rc = issue(c);
        if (rc != BGPU_OK) return rc;
    }
    for (size_t c = 0; c < chunks; ++c) {
        const int k = slot_of[c % kSlots];
        cudaError_t e = cudaEventSynchronize(g_ring.ev[k]);
        if (e != cudaSuccess) return status(e);
        g_ring.busy[k] = false;
        const size_t off = c * kSlot, len = std::min(kSlot, bytes - off);
        host_copy(static_cast<char*>(dst) + off, g_ring.host + (size_t)k * kSlot, len, false);
        if (c + kSlots < chunks) {
            rc = issue(c + kSlots);
            if (rc != BGPU_OK) return rc;
        }
    }
    return BGPU_OK;
}

void release_host_staging() {
    for (int k = 0; k < kSlots; ++k) {
        if (g_ring.ev[k]) {
            if (g_ring.busy[k]) cudaEventSynchronize(g_ring.ev[k]);
            cudaEventDestroy(g_ring.ev[k]);
        }
    }
    if (g_ring.host) cudaFreeHost(g_ring.host);
    g_ring = Ring{};
}

}  // namespace bgpu
