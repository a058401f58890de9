// Batched products: thousands of independent multiplies of uneven sizes in
// one CUDA-graph launch.
//
// The reference multiplies one pair at a time (each product internally
// threaded, src/mul/ntt_multithread.cpp:259-282); its binary-splitting and
// fast_pow callers produce many independent products per step
// (examples/pi.cpp:41-80).  A plan sorts the products of a batch into classes:
// products small enough for the schoolbook kernel (one CTA each), and NTT
// classes of equal transform length and squaring flag.  Every class runs as one
// set of launches with a grid slice per product, on its own branch of a CUDA
// graph so small classes overlap; the graph is built once per plan and
// replayed per run.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/bigint_b200.h"
#include "engine.h"

namespace bgpu {

// ---- plans -------------------------------------------------------------------

struct BatchClass {
    int log_n = 0;
    bool square = false;
    std::vector<uint32_t> members;  // product indices
    size_t desc_off = 0;            // into the ProductDesc device array
    size_t flags_off = 0, flags_words = 0;
    size_t scratch_off = 0;
};

}  // namespace bgpu

struct bgpu_batch_plan_s {
    int device = -1;
    size_t count = 0;
    std::vector<bgpu::BatchClass> classes;
    // every NTT class (and the small products) run in the four mixed-length
    // launches, one per pass
    bool mixed = false;
    bgpu::MixedSizes mixed_sizes{};
    std::vector<std::array<uint32_t, 4>> mixed_begin;  // per class, per pass
    std::vector<bgpu::SchoolDesc> school;  // schoolbook products
    std::vector<bgpu::SchoolDesc> kara;    // Karatsuba products
    void* d_mem = nullptr;  // descriptors, scratch, flags, tickets
    size_t d_bytes = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t launches = 0;
};

namespace bgpu {
namespace {

size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

int ceil_log2(uint64_t x) {
    int l = 0;
    while (((uint64_t)1 << l) < x) ++l;
    return l;
}

size_t ntt_scratch_bytes(int log_n, bool square) {
    const size_t nn = (size_t)1 << log_n;
    return al256((square ? 1 : 2) * (size_t)kNumPrimes * nn * 4) + al256(nn / 2 * 8) + al256(nn / 8 * 8);
}

void destroy_plan(bgpu_batch_plan_s* p) {
    if (!p) return;
    if (p->device >= 0) cudaSetDevice(p->device);
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    cudaFree(p->d_mem);
    delete p;
}

}  // namespace

// Record the plan's work on `st`: reset the carry-scan state, fork one branch
// per class onto the prepared streams, launch, and join back.
int batch_record(bgpu_batch_plan_s* p, cudaStream_t st, const EngineHooks& hooks,
                 const std::vector<cudaStream_t>& branches, const std::vector<cudaEvent_t>& joins,
                 cudaEvent_t fork) {
    char* base = static_cast<char*>(p->d_mem);
    const ProductDesc* d_descs = reinterpret_cast<const ProductDesc*>(base);
    size_t n_desc = 0, flag_words = 0;
    for (auto& c : p->classes) {
        n_desc += c.members.size();
        flag_words += c.flags_words;
    }
    const size_t mixed_off = al256(n_desc * sizeof(ProductDesc));
    const size_t school_off = mixed_off + al256((p->mixed ? p->classes.size() : 0) * sizeof(MixedClass));
    const size_t kara_off = school_off + al256(p->school.size() * sizeof(SchoolDesc));
    const size_t tick_off = kara_off + al256(p->kara.size() * sizeof(SchoolDesc));
    unsigned long long* tickets = reinterpret_cast<unsigned long long*>(base + tick_off);
    const size_t flags_base = tick_off + al256(std::max<size_t>(1, p->classes.size()) * 8);
    // Carry-scan state restarts every run: ticket counters and flag words at 0,
    // epoch 1 baked into the launches.
    cudaError_t e = cudaMemsetAsync(tickets, 0, std::max<size_t>(1, p->classes.size()) * 8, st);
    if (e == cudaSuccess && flag_words) e = cudaMemsetAsync(base + flags_base, 0, flag_words * 8, st);
    if (e == cudaSuccess) e = cudaEventRecord(fork, st);
    for (size_t i = 0; e == cudaSuccess && i < branches.size(); ++i) e = cudaStreamWaitEvent(branches[i], fork, 0);
    if (e != cudaSuccess) return BGPU_ERR_CUDA;
    uint32_t launches = 0;
    if (p->mixed) {
        // every class and the small products: four launches on the recording stream
        MixedArgs m{};
        m.classes = reinterpret_cast<const MixedClass*>(base + mixed_off);
        m.nclasses = (int)p->classes.size();
        for (size_t i = 0; i < p->classes.size(); ++i)
            for (int pass = 0; pass < 4; ++pass) m.begin[pass][i] = p->mixed_begin[i][pass];
        m.ticket = tickets;
        m.ticket_base = 0;
        m.epoch = 1;
        m.err = hooks.err;
        m.school = reinterpret_cast<const SchoolDesc*>(base + school_off);
        m.nschool = (uint32_t)p->school.size();
        m.kara = reinterpret_cast<const SchoolDesc*>(base + kara_off);
        m.nkara = (uint32_t)p->kara.size();
        if (launch_ntt_mixed(m, p->mixed_sizes, st) != cudaSuccess) return BGPU_ERR_CUDA;
        launches += kNttLaunches;
    }
    for (size_t ci = 0; !p->mixed && ci < p->classes.size(); ++ci) {
        const BatchClass& c = p->classes[ci];
        const int ps = prime_set_for(c.log_n);
        CarryLaunch cl;
        cl.ticket_base = 0;
        cl.epoch = 1;
        cl.ticket = tickets + ci;
        cl.err = hooks.err;
        e = launch_ntt_batch(kSlotEngine + ps, hooks.consts[ps], d_descs + c.desc_off,
                             (int)c.members.size(), c.square, c.log_n, kFmtLimb64, cl, branches[ci]);
        if (e != cudaSuccess) return BGPU_ERR_CUDA;
        launches += kNttLaunches;
    }
    size_t bi = p->mixed ? 0 : p->classes.size();
    if (!p->school.empty() && !p->mixed) {
        const SchoolDesc* d_school = reinterpret_cast<const SchoolDesc*>(base + school_off);
        if (launch_schoolbook_batch(d_school, (uint32_t)p->school.size(), branches[bi++]) != cudaSuccess)
            return BGPU_ERR_CUDA;
        launches += 1;
    }
    if (!p->kara.empty() && !p->mixed) {
        const SchoolDesc* d_kara = reinterpret_cast<const SchoolDesc*>(base + kara_off);
        if (launch_karatsuba_batch(d_kara, (uint32_t)p->kara.size(), branches[bi++]) != cudaSuccess)
            return BGPU_ERR_CUDA;
        launches += 1;
    }
    for (size_t i = 0; i < branches.size(); ++i) {
        if (cudaEventRecord(joins[i], branches[i]) != cudaSuccess ||
            cudaStreamWaitEvent(st, joins[i], 0) != cudaSuccess)
            return BGPU_ERR_CUDA;
    }
    p->launches = launches;
    return BGPU_OK;
}

int batch_plan_create(const bgpu_product* prods, size_t count, uint32_t flags, int device,
                      const EngineHooks& hooks, bgpu_batch_plan_s** out) {
    auto* p = new (std::nothrow) bgpu_batch_plan_s();
    if (!p) return BGPU_ERR_OOM;
    p->device = device;
    p->count = count;
    std::map<std::pair<int, bool>, size_t> index;
    for (size_t i = 0; i < count; ++i) {
        const bgpu_product& q = prods[i];
        if (!q.a || !q.b || !q.out || q.na == 0 || q.nb == 0) {
            destroy_plan(p);
            return BGPU_ERR_INVALID_ARG;
        }
        const bool square = q.a == q.b && q.na == q.nb;
        if (q.na + q.nb <= tuning().batch_schoolbook_max_limbs) {
            p->school.push_back(SchoolDesc{q.a, q.b, q.out, (uint32_t)q.na, (uint32_t)q.nb});
            continue;
        }
        if (q.na + q.nb <= tuning().batch_karatsuba_max_limbs && karatsuba_fits(q.na, q.nb)) {
            p->kara.push_back(SchoolDesc{q.a, q.b, q.out, (uint32_t)q.na, (uint32_t)q.nb});
            continue;
        }
        if (q.na + q.nb > ((size_t)1 << 31)) {
            destroy_plan(p);
            return BGPU_ERR_CAPACITY;
        }
        int ln = ceil_log2(2 * (uint64_t)(q.na + q.nb) - 1);
        if (ln < 5) ln = 5;
        if (!shape_supported_batch(ln, square)) {
            destroy_plan(p);
            return BGPU_ERR_CAPACITY;
        }
        auto key = std::make_pair(ln, square);
        auto it = index.find(key);
        if (it == index.end()) {
            it = index.emplace(key, p->classes.size()).first;
            p->classes.emplace_back();
            p->classes.back().log_n = ln;
            p->classes.back().square = square;
        }
        p->classes[it->second].members.push_back((uint32_t)i);
    }
    // Longest transforms first: in the mixed launches their CTAs, the longest
    // of each pass, start in the first wave and the short ones fill the tail.
    std::stable_sort(p->classes.begin(), p->classes.end(),
                     [](const BatchClass& x, const BatchClass& y) { return x.log_n > y.log_n; });
    // Layout: [ProductDesc...][MixedClass...][SchoolDesc: schoolbook...]
    //         [SchoolDesc: Karatsuba...][tickets][flags][scratch].
    size_t n_desc = 0, flag_words = 0, scratch = 0;
    for (auto& c : p->classes) {
        c.desc_off = n_desc;
        n_desc += c.members.size();
        c.flags_off = flag_words;
        c.flags_words = c.members.size() * carry_blocks((uint32_t)(((size_t)1 << c.log_n) / 8));
        flag_words += c.flags_words;
        c.scratch_off = scratch;
        scratch += c.members.size() * ntt_scratch_bytes(c.log_n, c.square);
    }
    // The mixed-length launches take every class when each qualifies and
    // there are several lengths, unless the caller asks for per-class launch
    // sets (BGPU_BATCH_PER_CLASS); a single length runs its own per-length
    // kernels (tuned for it, without the mixed launches' register budget):
    // a uniform batch of the decimal conversions' levels ran 5.6 -> 9.0 ms
    // per 1.26 M-digit print through the mixed launches.
#ifndef BGPU_MIXED_BATCH
#define BGPU_MIXED_BATCH 1
#endif
    p->mixed = BGPU_MIXED_BATCH && !(flags & BGPU_BATCH_PER_CLASS) && p->classes.size() >= 2 &&
               p->classes.size() <= (size_t)kMaxMixedClasses;
    for (auto& c : p->classes) p->mixed = p->mixed && mixed_class_ok(c.log_n, c.square);
    const size_t mixed_off = al256(n_desc * sizeof(ProductDesc));
    const size_t school_off = mixed_off + al256((p->mixed ? p->classes.size() : 0) * sizeof(MixedClass));
    const size_t kara_off = school_off + al256(p->school.size() * sizeof(SchoolDesc));
    const size_t tick_off = kara_off + al256(p->kara.size() * sizeof(SchoolDesc));
    const size_t flags_base = tick_off + al256(std::max<size_t>(1, p->classes.size()) * 8);
    const size_t scratch_base = flags_base + al256(flag_words * 8);
    p->d_bytes = scratch_base + scratch;
    if (cudaMalloc(&p->d_mem, p->d_bytes) != cudaSuccess) {
        cudaGetLastError();
        destroy_plan(p);
        return BGPU_ERR_OOM;
    }
    char* base = static_cast<char*>(p->d_mem);
    std::vector<ProductDesc> descs(n_desc);
    for (auto& c : p->classes) {
        const size_t nn = (size_t)1 << c.log_n;
        const size_t per = ntt_scratch_bytes(c.log_n, c.square);
        const size_t y_bytes = al256((c.square ? 1 : 2) * (size_t)kNumPrimes * nn * 4);
        for (size_t m = 0; m < c.members.size(); ++m) {
            const bgpu_product& q = prods[c.members[m]];
            char* sc = base + scratch_base + c.scratch_off + m * per;
            ProductDesc& d = descs[c.desc_off + m];
            d.op[0] = OperandDesc{q.a, (uint32_t)q.na, (uint32_t)(2 * q.na), kFmtLimb64};
            d.op[1] = c.square ? d.op[0] : OperandDesc{q.b, (uint32_t)q.nb, (uint32_t)(2 * q.nb), kFmtLimb64};
            d.y = reinterpret_cast<uint32_t*>(sc);
            d.chunks = reinterpret_cast<uint64_t*>(sc + y_bytes);
            d.spill = reinterpret_cast<uint64_t*>(sc + y_bytes + al256(nn / 2 * 8));
            d.flags = reinterpret_cast<uint64_t*>(base + flags_base) + c.flags_off +
                      m * carry_blocks((uint32_t)(nn / 8));
            d.out = q.out;
            d.out_cap = q.na + q.nb;
        }
    }
    cudaError_t e = cudaMemcpy(base, descs.data(), n_desc * sizeof(ProductDesc), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && p->mixed) {
        std::vector<MixedClassSpec> spec(p->classes.size());
        for (size_t i = 0; i < p->classes.size(); ++i) {
            const BatchClass& c = p->classes[i];
            spec[i] = MixedClassSpec{reinterpret_cast<const ProductDesc*>(base) + c.desc_off,
                                     (uint32_t)c.members.size(), c.log_n, c.square};
        }
        std::vector<MixedClass> mc(p->classes.size());
        if (mixed_fill(mc.data(), (int)mc.size(), spec.data(), kSlotEngine + 0, hooks.consts[0],
                       &p->mixed_sizes) != 0) {
            destroy_plan(p);
            return BGPU_ERR_INVALID_ARG;
        }
        for (auto& k : mc) k.inv.err = hooks.err;
        p->mixed_begin.resize(mc.size());
        for (size_t i = 0; i < mc.size(); ++i)
            for (int pass = 0; pass < 4; ++pass) p->mixed_begin[i][pass] = mc[i].begin[pass];
        e = cudaMemcpy(base + mixed_off, mc.data(), mc.size() * sizeof(MixedClass), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess && !p->school.empty())
        e = cudaMemcpy(base + school_off, p->school.data(), p->school.size() * sizeof(SchoolDesc),
                       cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !p->kara.empty())
        e = cudaMemcpy(base + kara_off, p->kara.data(), p->kara.size() * sizeof(SchoolDesc),
                       cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        destroy_plan(p);
        return BGPU_ERR_CUDA;
    }
    // Capture the whole batch into one graph (streams and events made first).
    const size_t nbranch = p->mixed ? 0 : p->classes.size() + (p->school.empty() ? 0 : 1) +
                                              (p->kara.empty() ? 0 : 1);
    std::vector<cudaStream_t> branches(nbranch, nullptr);
    std::vector<cudaEvent_t> joins(nbranch, nullptr);
    cudaStream_t cap = nullptr;
    cudaEvent_t fork = nullptr;
    int rc = BGPU_OK;
    if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&fork, cudaEventDisableTiming) != cudaSuccess)
        rc = BGPU_ERR_CUDA;
    for (size_t i = 0; rc == BGPU_OK && i < nbranch; ++i) {
        if (cudaStreamCreateWithFlags(&branches[i], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&joins[i], cudaEventDisableTiming) != cudaSuccess)
            rc = BGPU_ERR_CUDA;
    }
    cudaGraph_t g = nullptr;
    if (rc == BGPU_OK) {
        if (cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            rc = BGPU_ERR_CUDA;
        } else {
            rc = batch_record(p, cap, hooks, branches, joins, fork);
            const cudaError_t ec = cudaStreamEndCapture(cap, &g);
            if (rc == BGPU_OK && ec != cudaSuccess) rc = BGPU_ERR_CUDA;
        }
    }
    for (auto x : branches)
        if (x) cudaStreamDestroy(x);
    for (auto x : joins)
        if (x) cudaEventDestroy(x);
    if (fork) cudaEventDestroy(fork);
    if (cap) cudaStreamDestroy(cap);
    if (rc == BGPU_OK) {
        p->graph = g;
        if (cudaGraphInstantiate(&p->exec, g, 0) != cudaSuccess) rc = BGPU_ERR_CUDA;
    } else if (g) {
        cudaGraphDestroy(g);
    }
    if (rc != BGPU_OK) {
        cudaGetLastError();
        destroy_plan(p);
        return rc;
    }
    *out = p;
    return BGPU_OK;
}

int batch_plan_run(bgpu_batch_plan_s* p, cudaStream_t st) {
    if (!p || !p->exec) return BGPU_ERR_INVALID_ARG;
    return cudaGraphLaunch(p->exec, st) == cudaSuccess ? BGPU_OK : BGPU_ERR_CUDA;
}

void batch_plan_destroy(bgpu_batch_plan_s* p) { destroy_plan(p); }

uint32_t batch_plan_launches(const bgpu_batch_plan_s* p) { return p ? p->launches : 0; }
size_t batch_plan_classes(const bgpu_batch_plan_s* p) { return p ? p->classes.size() : 0; }

}  // namespace bgpu

// ---- product tree --------------------------------------------------------------
//
// The binary-splitting caller pattern (examples/pi.cpp:41-80; config "product
// tree"): n values multiplied pairwise level by level until one is left, the
// odd tail carried up unchanged.  Every level keeps its values at one width W
// (limbs, zero-padded), so a level is one uniform batch: a thread per product
// for W <= 4, then the batched schoolbook or Karatsuba kernel while 2W is
// within their tuned limits, then one NTT class.  Each level is a single set
// of launches; values stay on the GPU.

namespace bgpu {

template <int W>
__global__ void k_tree_small(const uint64_t* __restrict__ in, uint64_t* __restrict__ out, uint32_t m2) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m2) return;
    const uint64_t* a = in + (size_t)(2 * i) * W;
    const uint64_t* b = a + W;
    uint64_t r[2 * W];
#pragma unroll
    for (int k = 0; k < 2 * W; ++k) r[k] = 0;
#pragma unroll
    for (int x = 0; x < W; ++x) {
        uint64_t carry = 0;
#pragma unroll
        for (int y = 0; y < W; ++y) {
            const unsigned __int128 t = (unsigned __int128)a[x] * b[y] + r[x + y] + carry;
            r[x + y] = (uint64_t)t;
            carry = (uint64_t)(t >> 64);
        }
        r[x + W] = carry;
    }
    uint64_t* o = out + (size_t)i * 2 * W;
#pragma unroll
    for (int k = 0; k < 2 * W; ++k) o[k] = r[k];
}

// Copy the odd tail value (width W) into slot m2 of the next level (width 2W).
__global__ void k_tree_tail(const uint64_t* __restrict__ src, uint64_t* __restrict__ dst, uint32_t w) {
    for (uint32_t k = threadIdx.x; k < 2 * w; k += blockDim.x) dst[k] = k < w ? src[k] : 0;
}

namespace {

// One level of the tree: m values of width w become ceil(m/2) of width 2w.
struct TreeLevel {
    uint32_t m, m2;
    size_t w;
    int kind;  // 0: thread per product (w <= 4), 1: schoolbook, 2: Karatsuba, 3: NTT
    int log_n = 0;
    size_t desc_off = 0;  // bytes into the descriptor region
};

}  // namespace

int product_tree_device(const uint64_t* d_leaves, size_t n, uint64_t* d_out, size_t out_cap,
                        const EngineHooks& hooks, TreeArena* arena, cudaStream_t st, uint32_t* launches) {
    if (n == 0 || !arena) return BGPU_ERR_INVALID_ARG;
    // Final width: smallest power of two >= n limbs.
    size_t wfin = 1;
    while (wfin < n) wfin <<= 1;
    if (out_cap < wfin) return BGPU_ERR_OUT_CAPACITY;
    // Plan every level first: method, descriptor space, NTT scratch.
    const Tuning& tu = tuning();
    std::vector<TreeLevel> lv;
    size_t desc_bytes = 0, ntt_bytes = 0, flag_words = 0;
    for (size_t m = n, w = 1; m > 1; m = (m + 1) / 2, w *= 2) {
        TreeLevel L;
        L.m = (uint32_t)m;
        L.m2 = (uint32_t)(m / 2);
        L.w = w;
        if (w <= 4) {
            L.kind = 0;
        } else if (2 * w <= tu.batch_schoolbook_max_limbs) {
            L.kind = 1;
        } else if (2 * w <= tu.batch_karatsuba_max_limbs && karatsuba_fits(w, w)) {
            L.kind = 2;
        } else {
            L.kind = 3;
            while (((uint64_t)1 << L.log_n) < 4 * (uint64_t)w - 1) ++L.log_n;
            if (!shape_supported_batch(L.log_n, false)) return BGPU_ERR_CAPACITY;
            const size_t nn = (size_t)1 << L.log_n;
            ntt_bytes = std::max(ntt_bytes, (size_t)L.m2 * ntt_scratch_bytes(L.log_n, false));
            flag_words = std::max(flag_words, (size_t)L.m2 * carry_blocks((uint32_t)(nn / 8)));
        }
        if (L.kind == 1 || L.kind == 2) {
            L.desc_off = desc_bytes;
            desc_bytes += al256((size_t)L.m2 * sizeof(SchoolDesc));
        } else if (L.kind == 3) {
            L.desc_off = desc_bytes;
            desc_bytes += al256((size_t)L.m2 * sizeof(ProductDesc));
        }
        lv.push_back(L);
    }
    // Arena: [value buffer 0][value buffer 1][descriptors][ticket][flags][NTT scratch],
    // kept by the engine between calls (grow-only).
    const size_t cap_limbs = 2 * wfin + 16;
    const size_t buf_bytes = al256(cap_limbs * 8);
    const size_t off_desc = 2 * buf_bytes;
    const size_t off_ticket = off_desc + al256(desc_bytes);
    const size_t off_flags = off_ticket + 256;
    const size_t off_ntt = off_flags + al256(flag_words * 8);
    const size_t need = off_ntt + ntt_bytes;
    if (arena->bytes < need) {
        cudaStreamSynchronize(st);
        cudaFree(arena->ptr);
        arena->ptr = nullptr;
        arena->bytes = 0;
        if (cudaMalloc(&arena->ptr, need + need / 4) != cudaSuccess) {
            cudaGetLastError();
            return BGPU_ERR_OOM;
        }
        arena->bytes = need + need / 4;
    }
    char* base = static_cast<char*>(arena->ptr);
    uint64_t* buf[2] = {reinterpret_cast<uint64_t*>(base), reinterpret_cast<uint64_t*>(base + buf_bytes)};
    unsigned long long* ticket = reinterpret_cast<unsigned long long*>(base + off_ticket);
    uint64_t* flags = reinterpret_cast<uint64_t*>(base + off_flags);
    // Every level's descriptors, built on the host and copied in one go.
    std::vector<char> hd(desc_bytes);
    {
        int cur = 0;
        for (const TreeLevel& L : lv) {
            const uint64_t* in = buf[cur];
            uint64_t* out = buf[cur ^ 1];
            const size_t w = L.w;
            if (L.kind == 1 || L.kind == 2) {
                SchoolDesc* sd = reinterpret_cast<SchoolDesc*>(hd.data() + L.desc_off);
                for (uint32_t i = 0; i < L.m2; ++i)
                    sd[i] = SchoolDesc{in + (size_t)2 * i * w, in + (size_t)(2 * i + 1) * w,
                                       out + (size_t)2 * i * w, (uint32_t)w, (uint32_t)w};
            } else if (L.kind == 3) {
                ProductDesc* pd = reinterpret_cast<ProductDesc*>(hd.data() + L.desc_off);
                const size_t nn = (size_t)1 << L.log_n;
                const size_t per = ntt_scratch_bytes(L.log_n, false);
                const uint32_t bpp = carry_blocks((uint32_t)(nn / 8));
                const size_t y_bytes = al256(2 * (size_t)kNumPrimes * nn * 4);
                for (uint32_t i = 0; i < L.m2; ++i) {
                    char* sc = base + off_ntt + (size_t)i * per;
                    ProductDesc& d = pd[i];
                    d.op[0] = OperandDesc{in + (size_t)2 * i * w, (uint32_t)w, (uint32_t)(2 * w), kFmtLimb64};
                    d.op[1] = OperandDesc{in + (size_t)(2 * i + 1) * w, (uint32_t)w, (uint32_t)(2 * w), kFmtLimb64};
                    d.y = reinterpret_cast<uint32_t*>(sc);
                    d.chunks = reinterpret_cast<uint64_t*>(sc + y_bytes);
                    d.spill = reinterpret_cast<uint64_t*>(sc + y_bytes + al256(nn / 2 * 8));
                    d.flags = flags + (size_t)i * bpp;
                    d.out = out + (size_t)2 * i * w;
                    d.out_cap = 2 * w;
                }
            }
            cur ^= 1;
        }
    }
    cudaError_t e = cudaMemcpyAsync(buf[0], d_leaves, n * 8, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess && desc_bytes)
        e = cudaMemcpyAsync(base + off_desc, hd.data(), desc_bytes, cudaMemcpyHostToDevice, st);
    uint32_t nl = 0;
    int cur = 0;
    for (const TreeLevel& L : lv) {
        if (e != cudaSuccess) break;
        const uint64_t* in = buf[cur];
        uint64_t* out = buf[cur ^ 1];
        const size_t w = L.w;
        if (L.kind == 0) {
            const unsigned blocks = (L.m2 + 255) / 256;
            if (w == 1) k_tree_small<1><<<blocks, 256, 0, st>>>(in, out, L.m2);
            else if (w == 2) k_tree_small<2><<<blocks, 256, 0, st>>>(in, out, L.m2);
            else k_tree_small<4><<<blocks, 256, 0, st>>>(in, out, L.m2);
            e = cudaGetLastError();
            nl += 1;
        } else if (L.kind == 1 || L.kind == 2) {
            const SchoolDesc* d = reinterpret_cast<const SchoolDesc*>(base + off_desc + L.desc_off);
            e = L.kind == 2 ? launch_karatsuba_batch(d, L.m2, st) : launch_schoolbook_batch(d, L.m2, st);
            nl += 1;
        } else {
            // fresh carry-scan state for this level: ticket 0, flags 0, epoch 1
            const size_t nn = (size_t)1 << L.log_n;
            e = cudaMemsetAsync(ticket, 0, 8, st);
            if (e == cudaSuccess)
                e = cudaMemsetAsync(flags, 0, (size_t)L.m2 * carry_blocks((uint32_t)(nn / 8)) * 8, st);
            if (e == cudaSuccess) {
                CarryLaunch cl;
                cl.ticket_base = 0;
                cl.epoch = 1;
                cl.ticket = ticket;
                cl.err = hooks.err;
                const int ps = prime_set_for(L.log_n);
                e = launch_ntt_batch(kSlotEngine + ps, hooks.consts[ps],
                                     reinterpret_cast<const ProductDesc*>(base + off_desc + L.desc_off),
                                     (int)L.m2, false, L.log_n, kFmtLimb64, cl, st);
            }
            nl += kNttLaunches;
        }
        if (e == cudaSuccess && (L.m & 1)) {
            k_tree_tail<<<1, 256, 0, st>>>(in + (size_t)(L.m - 1) * w, out + (size_t)L.m2 * 2 * w, (uint32_t)w);
            e = cudaGetLastError();
            nl += 1;
        }
        cur ^= 1;
    }
    const size_t wlast = lv.empty() ? 1 : lv.back().w * 2;
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_out, buf[cur], wlast * 8, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // the host descriptors live until here
    if (launches) *launches = nl;
    return e == cudaSuccess ? BGPU_OK : BGPU_ERR_CUDA;
}

}  // namespace bgpu
