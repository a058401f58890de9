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
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/bigint_b200.h"
#include "engine.h"

namespace bgpu {

// ---- batched schoolbook ------------------------------------------------------

struct SchoolDesc {
    const uint64_t* a;
    const uint64_t* b;
    uint64_t* out;
    uint32_t na, nb;
};

constexpr int kSbThreads = 128;

// One CTA per product (na + nb <= kSchoolbookMaxLimbs): thread k owns output
// columns k, k + 128, ...; column sums are 192-bit, then one carry fold.
__global__ void __launch_bounds__(kSbThreads) k_schoolbook_batch(const SchoolDesc* descs) {
    __shared__ uint64_t sa[kSchoolbookMaxLimbs], sb[kSchoolbookMaxLimbs];
    __shared__ uint64_t c0[kSchoolbookMaxLimbs], c1[kSchoolbookMaxLimbs], c2[kSchoolbookMaxLimbs];
    const SchoolDesc d = descs[blockIdx.x];
    for (uint32_t i = threadIdx.x; i < d.na; i += kSbThreads) sa[i] = d.a[i];
    for (uint32_t i = threadIdx.x; i < d.nb; i += kSbThreads) sb[i] = d.b[i];
    __syncthreads();
    const uint32_t ncol = d.na + d.nb;
    for (uint32_t k = threadIdx.x; k < ncol; k += kSbThreads) {
        uint64_t x0 = 0, x1 = 0, x2 = 0;
        if (k + 1 < ncol) {
            const uint32_t i0 = k + 1 > d.nb ? k + 1 - d.nb : 0;
            const uint32_t i1 = k < d.na - 1 ? k : d.na - 1;
            for (uint32_t i = i0; i <= i1; ++i) {
                const uint64_t u = sa[i], v = sb[k - i];
                const uint64_t lo = u * v, hi = __umul64hi(u, v);
                x0 += lo;
                const uint64_t c = x0 < lo;
                const uint64_t t = x1 + hi;
                x2 += (t < x1);
                x1 = t + c;
                x2 += (x1 < c);
            }
        }
        c0[k] = x0, c1[k] = x1, c2[k] = x2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned __int128 carry = 0;
        for (uint32_t k = 0; k < ncol; ++k) {
            unsigned __int128 s = carry + c0[k];
            if (k >= 1) s += c1[k - 1];
            if (k >= 2) s += c2[k - 2];
            d.out[k] = (uint64_t)s;
            carry = s >> 64;
        }
    }
}

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
    std::vector<bgpu::SchoolDesc> school;
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
    const size_t school_off = al256(n_desc * sizeof(ProductDesc));
    const size_t tick_off = school_off + al256(p->school.size() * sizeof(SchoolDesc));
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
    for (size_t ci = 0; ci < p->classes.size(); ++ci) {
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
    if (!p->school.empty()) {
        const SchoolDesc* d_school = reinterpret_cast<const SchoolDesc*>(base + school_off);
        k_schoolbook_batch<<<(unsigned)p->school.size(), kSbThreads, 0, branches.back()>>>(d_school);
        if (cudaGetLastError() != cudaSuccess) return BGPU_ERR_CUDA;
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
    (void)flags;
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
        if (q.na + q.nb > ((size_t)1 << 31)) {
            destroy_plan(p);
            return BGPU_ERR_CAPACITY;
        }
        int ln = ceil_log2(2 * (uint64_t)(q.na + q.nb) - 1);
        if (ln < 5) ln = 5;
        if (!shape_supported(ln, square)) {
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
    // Layout: [ProductDesc...][SchoolDesc...][tickets][flags][scratch].
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
    const size_t school_off = al256(n_desc * sizeof(ProductDesc));
    const size_t tick_off = school_off + al256(p->school.size() * sizeof(SchoolDesc));
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
    if (e == cudaSuccess && !p->school.empty())
        e = cudaMemcpy(base + school_off, p->school.data(), p->school.size() * sizeof(SchoolDesc),
                       cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        destroy_plan(p);
        return BGPU_ERR_CUDA;
    }
    // Capture the whole batch into one graph (streams and events made first).
    const size_t nbranch = p->classes.size() + (p->school.empty() ? 0 : 1);
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
// for W <= 4, the batched schoolbook kernel while 2W <= 256 limbs, then one
// NTT class.  Each level is a single set of launches; values stay on the GPU.

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

int product_tree_device(const uint64_t* d_leaves, size_t n, uint64_t* d_out, size_t out_cap,
                        const EngineHooks& hooks, cudaStream_t st, uint32_t* launches) {
    if (n == 0) return BGPU_ERR_INVALID_ARG;
    // Final width: smallest power of two >= n limbs.
    size_t wfin = 1;
    while (wfin < n) wfin <<= 1;
    if (out_cap < wfin) return BGPU_ERR_OUT_CAPACITY;
    const size_t cap_limbs = 2 * wfin + 16;
    uint64_t *buf[2] = {nullptr, nullptr};
    void* scratch = nullptr;
    void* descs = nullptr;
    size_t scratch_bytes = 0, desc_bytes = 0;
    uint32_t nl = 0;
    auto fail = [&](int rc) {
        cudaStreamSynchronize(st);
        cudaFree(buf[0]);
        cudaFree(buf[1]);
        cudaFree(scratch);
        cudaFree(descs);
        return rc;
    };
    if (cudaMalloc(&buf[0], cap_limbs * 8) != cudaSuccess || cudaMalloc(&buf[1], cap_limbs * 8) != cudaSuccess) {
        cudaGetLastError();
        return fail(BGPU_ERR_OOM);
    }
    if (cudaMemcpyAsync(buf[0], d_leaves, n * 8, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return fail(BGPU_ERR_CUDA);
    size_t m = n, w = 1;
    int cur = 0;
    std::vector<SchoolDesc> sd;
    std::vector<ProductDesc> pd;
    while (m > 1) {
        const uint32_t m2 = (uint32_t)(m / 2);
        const uint64_t* in = buf[cur];
        uint64_t* out = buf[cur ^ 1];
        cudaError_t e = cudaSuccess;
        if (w <= 4) {
            const unsigned blocks = (m2 + 255) / 256;
            if (w == 1) k_tree_small<1><<<blocks, 256, 0, st>>>(in, out, m2);
            else if (w == 2) k_tree_small<2><<<blocks, 256, 0, st>>>(in, out, m2);
            else k_tree_small<4><<<blocks, 256, 0, st>>>(in, out, m2);
            e = cudaGetLastError();
            nl += 1;
        } else if (2 * w <= tuning().batch_schoolbook_max_limbs) {
            sd.resize(m2);
            for (uint32_t i = 0; i < m2; ++i)
                sd[i] = SchoolDesc{in + (size_t)2 * i * w, in + (size_t)(2 * i + 1) * w, out + (size_t)2 * i * w,
                                   (uint32_t)w, (uint32_t)w};
            const size_t need = m2 * sizeof(SchoolDesc);
            if (need > desc_bytes) {
                cudaStreamSynchronize(st);
                cudaFree(descs);
                descs = nullptr;
                if (cudaMalloc(&descs, need) != cudaSuccess) return fail(BGPU_ERR_OOM);
                desc_bytes = need;
            }
            // synchronous copy: the host array is reused by the next level
            e = cudaMemcpyAsync(descs, sd.data(), need, cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e == cudaSuccess) {
                k_schoolbook_batch<<<m2, kSbThreads, 0, st>>>(static_cast<const SchoolDesc*>(descs));
                e = cudaGetLastError();
            }
            nl += 1;
        } else {
            int ln = 0;
            while (((uint64_t)1 << ln) < 4 * (uint64_t)w - 1) ++ln;
            if (!shape_supported(ln, false)) return fail(BGPU_ERR_CAPACITY);
            const size_t nn = (size_t)1 << ln;
            const size_t per = ntt_scratch_bytes(ln, false);
            const uint32_t bpp = carry_blocks((uint32_t)(nn / 8));
            const size_t flag_bytes = al256((size_t)m2 * bpp * 8) + 256;
            const size_t need_s = m2 * per + flag_bytes;
            if (need_s > scratch_bytes) {
                cudaStreamSynchronize(st);
                cudaFree(scratch);
                scratch = nullptr;
                if (cudaMalloc(&scratch, need_s) != cudaSuccess) return fail(BGPU_ERR_OOM);
                scratch_bytes = need_s;
            }
            char* sbase = static_cast<char*>(scratch);
            uint64_t* flags = reinterpret_cast<uint64_t*>(sbase + m2 * per);
            unsigned long long* ticket = reinterpret_cast<unsigned long long*>(sbase + m2 * per + al256((size_t)m2 * bpp * 8));
            const size_t y_bytes = al256(2 * (size_t)kNumPrimes * nn * 4);
            pd.resize(m2);
            for (uint32_t i = 0; i < m2; ++i) {
                char* sc = sbase + (size_t)i * per;
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
            const size_t need = m2 * sizeof(ProductDesc);
            if (need > desc_bytes) {
                cudaStreamSynchronize(st);
                cudaFree(descs);
                descs = nullptr;
                if (cudaMalloc(&descs, need) != cudaSuccess) return fail(BGPU_ERR_OOM);
                desc_bytes = need;
            }
            e = cudaMemcpyAsync(descs, pd.data(), need, cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            // fresh carry-scan state for this level: ticket 0, flags 0, epoch 1
            if (e == cudaSuccess) e = cudaMemsetAsync(ticket, 0, 8, st);
            if (e == cudaSuccess) e = cudaMemsetAsync(flags, 0, (size_t)m2 * bpp * 8, st);
            if (e == cudaSuccess) {
                CarryLaunch cl;
                cl.ticket_base = 0;
                cl.epoch = 1;
                cl.ticket = ticket;
                cl.err = hooks.err;
                if (e == cudaSuccess)
                    e = launch_ntt_batch(kSlotEngine + prime_set_for(ln), hooks.consts[prime_set_for(ln)],
                                         static_cast<const ProductDesc*>(descs), (int)m2, false, ln,
                                         kFmtLimb64, cl, st);
            }
            nl += kNttLaunches;
        }
        if (e == cudaSuccess && (m & 1)) {
            k_tree_tail<<<1, 256, 0, st>>>(in + (m - 1) * w, out + (size_t)m2 * 2 * w, (uint32_t)w);
            e = cudaGetLastError();
            nl += 1;
        }
        if (e != cudaSuccess) return fail(BGPU_ERR_CUDA);
        m = (m + 1) / 2;
        w *= 2;
        cur ^= 1;
    }
    cudaError_t e = cudaMemcpyAsync(d_out, buf[cur], w * 8, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (launches) *launches = nl;
    const int rc = e == cudaSuccess ? BGPU_OK : BGPU_ERR_CUDA;
    cudaFree(buf[0]);
    cudaFree(buf[1]);
    cudaFree(scratch);
    cudaFree(descs);
    return rc;
}

}  // namespace bgpu
