// common.cuh -- shared internals of libb2m: context, device workspaces, error plumbing,
// tensor-map encoding and the small PTX helpers used by the sm_100a kernels.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <functional>
#include <map>
#include <mutex>
#include <utility>
#include <tuple>
#include <type_traits>
#include <string>
#include <vector>

#include "../../include/b2m.h"

namespace b2m {

// ------------------------------------------------------------------ device status words
// Every context owns a small device array of int32 status words.  Kernels that can fail
// (singular pivot, bounded wait that gave up) write here; the host reads it after the call.
enum StatusWord : int {
    kInfo = 0,      // 0 ok, 1 singular (first singular pivot stops the factorisation)
    kTimeout = 1,   // nonzero: some bounded wait gave up; value = site id
    kIrIters = 2,   // refinement iterations done (mixed solve)
    kIrState = 3,   // refinement state: 0 converged, 1 stalled, 2 diverged
    kNumStatus = 8
};

// ------------------------------------------------------------------ workspace slots
enum WsSlot : int {
    kWsMatA = 0,   // device copy of A (host API) / LU factors
    kWsMatB,       // device copy of B / X
    kWsMatC,       // device copy of C / scratch
    kWsMatD,       // extra (FP32 LU, Ozaki slices, ...)
    kWsPiv,        // pivots and permutation
    kWsSmall,      // norms, small vectors
    kWsE,
    kWsF,
    kWsG,          // the mixed solve's X when the caller's buffer cannot be used directly
    kWsH,
    kWsPmap,       // row maps of the blocked FP64 LU's outer panels
    kWsTri,        // the FP64 blocked sweeps' diagonal inverses, coupling blocks and published blocks
    kNumWs
};

// kernel classes for the optional event profiler (b2m_profile / b2m_profile_read).  The work
// recorded with each launch is algorithmic: FLOPs for the tensor-core GEMM classes (gemm_f64,
// gemm_tc -- for gemm_tc the MMA passes of a split mode are counted), bytes that must cross HBM for
// every other class (panel, row moves, triangular solves, the residual under `other`).
enum KernelClass : int { kClsGemm = 0, kClsPanel, kClsSwap, kClsTrsm, kClsTcGemm, kClsSolve, kClsOther, kNumCls };

struct Prof {
    bool on = false;
    std::vector<cudaEvent_t> ev[kNumCls];  // start/end pairs
    size_t used[kNumCls] = {};
    double work[kNumCls] = {};             // algorithmic flops (or bytes) recorded with the launches
};

// key of a captured launch sequence: (kind, pointers and sizes baked into the graph)
typedef std::tuple<int, const void*, const void*, const void*, const void*, int64_t, int64_t, int64_t, int64_t>
    GraphKey;
struct GraphEntry {
    cudaGraphExec_t exec = nullptr;
    int64_t launches = 0;
    uint64_t last_use = 0;
};

// tile shape of the batched solve, chosen by its autotuner (batched.cu)
struct BatchTune {
    int small_n;      // systems of order <= small_n run on groups of group_warps warps
    int group_warps;
    int pw_large;     // panel widths of the two size buckets
    int pw_small;
    int big_warps;    // warps per system of order > small_n (8: the whole CTA, 4: two per CTA)
    float ms;         // measured time of the whole batch with this shape
};

// one progress report, enqueued as a host function behind the panel it reports on
struct ProgressNote {
    b2m_progress_fn fn;
    void* user;
    int32_t percent;
};

struct Ctx {
    int device = 0;
    int num_sms = 148;
    int sweep_ctas = -1;  // co-resident CTAs of the persistent refinement sweep (-1: not queried yet)
    int chain_clusters = -1;  // co-resident 8-CTA clusters of the chained sweep (0: unusable, -1: not probed)
    int chain_clusters4 = -1; // the same for 4-CTA clusters
    int chain_probe_why = 0;  // why it is unusable: step * 1000 + CUDA error (b2m_ctx_info)
    int dsweep_ctas = -1;     // co-resident CTAs of the FP64 blocked sweep (-1: not queried yet)
    int64_t wait_limit = -1;  // polls of the refinement sweeps' bounded waits (-1: the built-in limit)
    size_t smem_optin = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    int32_t* d_status = nullptr;     // kNumStatus words
    int32_t* h_status = nullptr;     // pinned mirror
    void* ws[kNumWs] = {};
    size_t ws_bytes[kNumWs] = {};
    // run_graph's own capture is in progress: a workspace slot that must grow is recorded here
    // (cudaMalloc is not allowed under capture) and the capture is redone after the allocation
    bool capturing = false;
    int ws_pending_slot = -1;
    size_t ws_pending_bytes = 0;
    void* h_pinned = nullptr;        // pinned staging for host-buffer calls
    size_t h_pinned_bytes = 0;
    int64_t launches = 0;
    Prof prof;
    bool use_graphs = true;
    std::map<GraphKey, GraphEntry> graphs;
    uint64_t graph_clock = 0;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaStream_t side_stream = nullptr;                  // look-ahead trailing updates of the FP32 LU
    cudaEvent_t ev_side_fork = nullptr, ev_side_join = nullptr;
    cudaStream_t leaf_stream = nullptr;  // FP64 LU: a leaf's work on its outer panel beyond the next leaf
    cudaEvent_t ev_leaf_panel = nullptr, ev_leaf_side = nullptr;
    int chain_priority = 0;                               // stream priority of the panel kernels
    bool launch_hi = false;  // launch_k adds the launch attribute `priority = chain_priority` (PriorityScope)
    std::string last_error;
    std::mutex mtx;
    b2m_progress_fn progress = nullptr;          // LU progress callback (b2m_set_progress)
    void* progress_user = nullptr;
    std::vector<ProgressNote> progress_notes;    // host-function payloads of the current call
    std::map<uint64_t, BatchTune> batch_tunes;  // per batch plan
    uint64_t batch_plan_sig = 0;                 // plan whose metadata is on the device now
    void* batch_plan_dev = nullptr;
};

// records a message and returns the status (for `return fail(ctx, ...)`)
int32_t fail(Ctx* ctx, int32_t status, const char* fmt, ...);

// internal status (never returned by an entry point): a workspace slot must grow while run_graph
// captures; run_graph allocates it and captures again
constexpr int32_t kWsRetry = -1000;

// an entry point's hold on its context: takes the context's mutex and clears a launch error that
// earlier work in this thread left behind (a non-sticky error such as a failed launch of someone
// else's kernel), so that the launch checks of this call report this call's errors only
struct CallLock {
    std::lock_guard<std::mutex> lk;
    explicit CallLock(Ctx* ctx) : lk(ctx->mtx) { (void)cudaGetLastError(); }
};

#define B2M_CU(ctx, call)                                                                          \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return ::b2m::fail((ctx), B2M_ERR_CUDA, "%s failed: %s (%s:%d)", #call,                \
                               cudaGetErrorString(e_), __FILE__, __LINE__);                        \
    } while (0)

#define B2M_TRY(expr)                                                                              \
    do {                                                                                           \
        int32_t s_ = (expr);                                                                       \
        if (s_ != B2M_OK) return s_;                                                               \
    } while (0)

// after a launch: count it and surface launch-configuration errors
#define B2M_LAUNCHED(ctx)                                                                          \
    do {                                                                                           \
        (ctx)->launches++;                                                                         \
        cudaError_t e_ = cudaGetLastError();                                                       \
        if (e_ != cudaSuccess)                                                                     \
            return ::b2m::fail((ctx), B2M_ERR_CUDA, "kernel launch failed: %s (%s:%d)",            \
                               cudaGetErrorString(e_), __FILE__, __LINE__);                        \
    } while (0)

// Launches `kern` on `st`; while a PriorityScope marks the launches as the critical path, with the
// launch attribute priority = ctx->chain_priority (graphs keep it per node: they are instantiated
// with per-node priorities), so that they take SMs ahead of a concurrent look-ahead update.
template <typename... KArgs, typename... Args>
cudaError_t launch_k(Ctx* ctx, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                     Args&&... args) {
    cudaLaunchConfig_t c{};
    c.gridDim = grid;
    c.blockDim = block;
    c.dynamicSmemBytes = smem;
    c.stream = st;
    cudaLaunchAttribute at[1];
    if (ctx->launch_hi) {
        at[0].id = cudaLaunchAttributePriority;
        at[0].val.priority = ctx->chain_priority;
        c.attrs = at;
        c.numAttrs = 1;
    }
    return cudaLaunchKernelEx(&c, kern, std::forward<Args>(args)...);
}
// marks (hi = true) or unmarks the launches issued while it lives
struct PriorityScope {
    Ctx* ctx;
    bool prev;
    PriorityScope(Ctx* c, bool hi) : ctx(c), prev(c->launch_hi) { c->launch_hi = hi; }
    ~PriorityScope() { ctx->launch_hi = prev; }
};

// Event profiler: brackets one launch on stream `st` (no-ops unless enabled).
void prof_begin(Ctx* ctx, cudaStream_t st, int cls);
void prof_end(Ctx* ctx, cudaStream_t st, int cls, double work);

// Runs `issue(stream)` -- a launch sequence whose shape depends only on `key` -- through a cached
// CUDA graph: the first call captures and instantiates it, later calls replay it.  The legacy
// default stream cannot be captured, so the graph then runs on the context's own stream, joined
// to `st` with events both ways.  Falls back to eager launches while profiling.
int32_t run_graph(Ctx* ctx, cudaStream_t st, const GraphKey& key, const std::function<int32_t(cudaStream_t)>& issue);

// Per-device flag for one-time launch set-up (cudaFuncSetAttribute applies to the current device
// only, and a process may drive several devices).  `key` is the kernel's address, `tag` tells apart
// several flags of one kernel (e.g. a cluster size).  The returned atomic starts at 0 and lives until
// exit; setting an attribute twice is harmless, so callers test, set the attributes, then store 1.
std::atomic<int>& device_flag(const void* key, int tag, int device);

// grows workspace slot `slot` to at least `bytes` (never shrinks); 256-byte aligned
int32_t ws_get(Ctx* ctx, int slot, size_t bytes, void** out);
int32_t pinned_get(Ctx* ctx, size_t bytes, void** out);

// ------------------------------------------------------------------ tensor maps
// cuTensorMapEncodeTiled through the runtime's driver entry point (no -lcuda needed).
int32_t encode_tmap_2d(Ctx* ctx, CUtensorMap* map, CUtensorMapDataType dtype, int elem_bytes, const void* base,
                       uint64_t inner, uint64_t outer, uint64_t row_stride_bytes, uint32_t box_inner,
                       uint32_t box_outer, CUtensorMapSwizzle swizzle);

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// ------------------------------------------------------------------ device helpers
// Bounded waits: every spin in this library gives up after this many polls and reports
// B2M_ERR_TIMEOUT through the status words instead of hanging the GPU.
constexpr uint32_t kSpinLimit = 1u << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// bulk (non-tensor) asynchronous copy of `bytes` (a multiple of 16, both addresses 16-byte
// aligned) from global memory into this CTA's shared memory, completing on `bar`
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// returns false (and flags `timeout_word`) if the phase never completed
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int32_t* timeout_word, int site) {
    for (uint32_t i = 0; i < kSpinLimit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    if (timeout_word) atomicExch(timeout_word, site);
    return false;
}

// A strided copy loop "for e = t; e < total; e += NT: put(e, get(e))" whose loads are issued CH at
// a time before any of their results is used, so that a loop of global loads feeding shared
// stores pays one memory latency per CH elements instead of one per element.  get(e) is only
// called for e < total.
template <int NT, int CH, typename T, typename Get, typename Put>
__device__ __forceinline__ void batched_copy(int t, int total, Get get, Put put) {
    for (int base = t; base < total; base += NT * CH) {
        T v[CH];
#pragma unroll
        for (int i = 0; i < CH; ++i) {
            const int e = base + NT * i;
            v[i] = e < total ? get(e) : T(0);
        }
#pragma unroll
        for (int i = 0; i < CH; ++i) {
            const int e = base + NT * i;
            if (e < total) put(e, v[i]);
        }
    }
}

// 16-byte asynchronous global -> shared copy (src_bytes < 16 zero-fills the rest), its commit
// group and the wait for all but N groups.
__device__ __forceinline__ void cp_async16(void* dst, const void* src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Distributed shared memory of a thread-block cluster: the address of `local` in CTA `rank`, a
// 16-byte store into another CTA's shared memory completing on its mbarrier, and a wait on this
// CTA's mbarrier that acquires at cluster scope.
__device__ __forceinline__ uint32_t map_rank(const void* local, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(smem_u32(local)), "r"(rank));
    return r;
}

__device__ __forceinline__ void st_async16(uint32_t raddr, uint4 v, uint32_t rbar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.b32 [%0], {%1, %2, %3, %4}, [%5];\n" ::"r"(
                     raddr),
                 "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w), "r"(rbar)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait_cluster(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// 2-D tiled TMA load (no multicast) into shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_2d(void* smem_dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];\n" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
__host__ __device__ inline int64_t round_up(int64_t a, int64_t b) { return ceil_div(a, b) * b; }

}  // namespace b2m
