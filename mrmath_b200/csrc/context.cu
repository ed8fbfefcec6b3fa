// context.cu -- context lifetime, workspaces, error strings and tensor-map encoding.
#include <cstdarg>
#include <cstring>

#include "common.cuh"

namespace b2m {

int32_t fail(Ctx* ctx, int32_t status, const char* fmt, ...) {
    if (ctx) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        ctx->last_error = buf;
    }
    return status;
}

std::atomic<int>& device_flag(const void* key, int tag, int device) {
    static std::mutex m;
    static std::map<std::tuple<const void*, int, int>, std::atomic<int>> flags;  // nodes never move
    std::lock_guard<std::mutex> lk(m);
    return flags[std::make_tuple(key, tag, device)];
}

int32_t ws_get(Ctx* ctx, int slot, size_t bytes, void** out) {
    bytes = (size_t)round_up((int64_t)std::max<size_t>(bytes, 256), 256);
    if (ctx->ws_bytes[slot] < bytes && ctx->capturing) {
        ctx->ws_pending_slot = slot;
        ctx->ws_pending_bytes = bytes;
        return kWsRetry;
    }
    if (ctx->ws_bytes[slot] < bytes) {
        if (ctx->ws[slot]) {
            // the buffer may still be in use by queued work, and captured graphs hold its address:
            // drain both streams and drop every cached graph before freeing it
            B2M_CU(ctx, cudaStreamSynchronize(ctx->stream));
            if (ctx->own_stream) B2M_CU(ctx, cudaStreamSynchronize(ctx->own_stream));
            if (ctx->side_stream) B2M_CU(ctx, cudaStreamSynchronize(ctx->side_stream));
            if (ctx->leaf_stream) B2M_CU(ctx, cudaStreamSynchronize(ctx->leaf_stream));
            for (auto& g : ctx->graphs) cudaGraphExecDestroy(g.second.exec);
            ctx->graphs.clear();
            B2M_CU(ctx, cudaFree(ctx->ws[slot]));
            ctx->ws[slot] = nullptr;
            ctx->ws_bytes[slot] = 0;
        }
        if (cudaMalloc(&ctx->ws[slot], bytes) != cudaSuccess) {
            cudaGetLastError();
            return fail(ctx, B2M_ERR_ALLOC, "cudaMalloc(%zu) failed for workspace slot %d", bytes, slot);
        }
        ctx->ws_bytes[slot] = bytes;
    }
    *out = ctx->ws[slot];
    return B2M_OK;
}

int32_t pinned_get(Ctx* ctx, size_t bytes, void** out) {
    if (ctx->h_pinned_bytes < bytes) {
        if (ctx->h_pinned) {
            B2M_CU(ctx, cudaStreamSynchronize(ctx->stream));
            cudaFreeHost(ctx->h_pinned);
            ctx->h_pinned = nullptr;
            ctx->h_pinned_bytes = 0;
        }
        if (cudaMallocHost(&ctx->h_pinned, bytes) != cudaSuccess) {
            cudaGetLastError();
            return fail(ctx, B2M_ERR_ALLOC, "cudaMallocHost(%zu) failed", bytes);
        }
        ctx->h_pinned_bytes = bytes;
    }
    *out = ctx->h_pinned;
    return B2M_OK;
}

void prof_begin(Ctx* ctx, cudaStream_t st, int cls) {
    Prof& p = ctx->prof;
    if (!p.on) return;
    if (p.used[cls] + 2 > p.ev[cls].size()) {
        for (int i = 0; i < 64; ++i) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return;
            p.ev[cls].push_back(e);
        }
    }
    cudaEventRecord(p.ev[cls][p.used[cls]], st);
}

void prof_end(Ctx* ctx, cudaStream_t st, int cls, double work) {
    Prof& p = ctx->prof;
    if (!p.on || p.used[cls] + 2 > p.ev[cls].size()) return;
    cudaEventRecord(p.ev[cls][p.used[cls] + 1], st);
    p.used[cls] += 2;
    p.work[cls] += work;
}

int32_t run_graph(Ctx* ctx, cudaStream_t st, const GraphKey& key, const std::function<int32_t(cudaStream_t)>& issue) {
    if (!ctx->use_graphs || ctx->prof.on || ctx->progress) return issue(st);
    cudaStreamCaptureStatus cs_status = cudaStreamCaptureStatusNone;
    if (st != nullptr && st != cudaStreamLegacy) {
        B2M_CU(ctx, cudaStreamIsCapturing(st, &cs_status));
        if (cs_status != cudaStreamCaptureStatusNone) return issue(st);  // the caller is capturing: join it
    }
    const bool fork = (st == nullptr || st == cudaStreamLegacy || st == cudaStreamPerThread);
    cudaStream_t gs = fork ? ctx->own_stream : st;
    auto it = ctx->graphs.find(key);
    if (it == ctx->graphs.end()) {
        if (ctx->graphs.size() >= 32) {  // evict the least recently used graph
            auto lru = ctx->graphs.begin();
            for (auto g = ctx->graphs.begin(); g != ctx->graphs.end(); ++g)
                if (g->second.last_use < lru->second.last_use) lru = g;
            B2M_CU(ctx, cudaStreamSynchronize(gs));
            cudaGraphExecDestroy(lru->second.exec);
            ctx->graphs.erase(lru);
        }
        cudaGraph_t g = nullptr;
        const int64_t l0 = ctx->launches;
        // a capture that needs a larger workspace slot is abandoned, the slot allocated outside
        // capture, and the capture redone (at most once per slot)
        for (int attempt = 0;; ++attempt) {
            B2M_CU(ctx, cudaStreamBeginCapture(gs, cudaStreamCaptureModeThreadLocal));
            ctx->capturing = true;
            const int32_t r = issue(gs);
            ctx->capturing = false;
            const cudaError_t ce = cudaStreamEndCapture(gs, &g);
            if (r != B2M_OK || ce != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                g = nullptr;
                (void)cudaGetLastError();  // an abandoned capture leaves no error for later calls
                ctx->launches = l0;
            }
            if (r == kWsRetry && attempt < 2 * kNumWs) {
                void* p = nullptr;
                B2M_TRY(ws_get(ctx, ctx->ws_pending_slot, ctx->ws_pending_bytes, &p));
                continue;
            }
            if (r == kWsRetry) return fail(ctx, B2M_ERR_ALLOC, "workspace kept growing under capture");
            if (r != B2M_OK) return r;
            if (ce != cudaSuccess)
                return fail(ctx, B2M_ERR_CUDA, "stream capture failed: %s", cudaGetErrorString(ce));
            break;
        }
        GraphEntry e;
        // per-node priorities: the LU's panel kernels are launched with the highest priority so that
        // they take SMs ahead of a concurrent trailing GEMM (a graph otherwise ignores them)
        const cudaError_t ie = cudaGraphInstantiateWithFlags(&e.exec, g, cudaGraphInstantiateFlagUseNodePriority);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) return fail(ctx, B2M_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(ie));
        e.launches = ctx->launches - l0;
        ctx->launches = l0;
        it = ctx->graphs.emplace(key, e).first;
    }
    it->second.last_use = ++ctx->graph_clock;
    if (fork) {
        if (!ctx->ev_fork) {
            B2M_CU(ctx, cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
            B2M_CU(ctx, cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming));
        }
        B2M_CU(ctx, cudaEventRecord(ctx->ev_fork, st));
        B2M_CU(ctx, cudaStreamWaitEvent(gs, ctx->ev_fork, 0));
    }
    B2M_CU(ctx, cudaGraphLaunch(it->second.exec, gs));
    if (fork) {
        B2M_CU(ctx, cudaEventRecord(ctx->ev_join, gs));
        B2M_CU(ctx, cudaStreamWaitEvent(st, ctx->ev_join, 0));
    }
    ctx->launches += it->second.launches;
    return B2M_OK;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn get_encode_fn(Ctx* ctx) {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    if (!fn) fail(ctx, B2M_ERR_CUDA, "cuTensorMapEncodeTiled entry point not available");
    return fn;
}

int32_t encode_tmap_2d(Ctx* ctx, CUtensorMap* map, CUtensorMapDataType dtype, int elem_bytes, const void* base,
                       uint64_t inner, uint64_t outer, uint64_t row_stride_bytes, uint32_t box_inner,
                       uint32_t box_outer, CUtensorMapSwizzle swizzle) {
    EncodeTiledFn fn = get_encode_fn(ctx);
    if (!fn) return B2M_ERR_CUDA;
    if (!aligned16(base) || (row_stride_bytes & 15u) != 0)
        return fail(ctx, B2M_ERR_DIM, "tensor map needs a 16-byte aligned base and stride (stride %llu)",
                    (unsigned long long)row_stride_bytes);
    cuuint64_t dims[2] = {inner, outer};
    cuuint64_t strides[1] = {row_stride_bytes};
    cuuint32_t box[2] = {box_inner, box_outer};
    cuuint32_t estr[2] = {1, 1};
    (void)elem_bytes;
    CUresult r = fn(map, dtype, 2, const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return fail(ctx, B2M_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d): dims %llu x %llu stride %llu box %u x %u",
                    (int)r, (unsigned long long)inner, (unsigned long long)outer,
                    (unsigned long long)row_stride_bytes, box_inner, box_outer);
    return B2M_OK;
}

}  // namespace b2m

using b2m::Ctx;

extern "C" int32_t b2m_create(int32_t device, b2m_ctx** out) {
    if (!out) return B2M_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return B2M_ERR_CUDA;
    }
    Ctx* ctx = new Ctx();
    ctx->device = device;
    if (cudaSetDevice(device) != cudaSuccess) { delete ctx; return B2M_ERR_CUDA; }
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, device);
    ctx->num_sms = prop.multiProcessorCount;
    ctx->smem_optin = prop.sharedMemPerBlockOptin;
    if (prop.major != 10) {
        delete ctx;
        return B2M_ERR_UNSUPPORTED;  // built for sm_100a only
    }
    if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return B2M_ERR_CUDA;
    }
    ctx->stream = ctx->own_stream;
    if (cudaMalloc(&ctx->d_status, b2m::kNumStatus * sizeof(int32_t)) != cudaSuccess ||
        cudaMallocHost(&ctx->h_status, b2m::kNumStatus * sizeof(int32_t)) != cudaSuccess) {
        cudaGetLastError();
        delete ctx;
        return B2M_ERR_ALLOC;
    }
    cudaMemset(ctx->d_status, 0, b2m::kNumStatus * sizeof(int32_t));
    std::memset(ctx->h_status, 0, b2m::kNumStatus * sizeof(int32_t));
    cudaDeviceSynchronize();
    *out = reinterpret_cast<b2m_ctx*>(ctx);
    return B2M_OK;
}

extern "C" int32_t b2m_destroy(b2m_ctx* h) {
    Ctx* ctx = reinterpret_cast<Ctx*>(h);
    if (!ctx) return B2M_ERR_ARG;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (int i = 0; i < b2m::kNumWs; ++i)
        if (ctx->ws[i]) cudaFree(ctx->ws[i]);
    if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
    if (ctx->d_status) cudaFree(ctx->d_status);
    if (ctx->h_status) cudaFreeHost(ctx->h_status);
    if (ctx->side_stream) cudaStreamDestroy(ctx->side_stream);
    if (ctx->leaf_stream) cudaStreamDestroy(ctx->leaf_stream);
    if (ctx->ev_leaf_panel) cudaEventDestroy(ctx->ev_leaf_panel);
    if (ctx->ev_leaf_side) cudaEventDestroy(ctx->ev_leaf_side);
    if (ctx->ev_side_fork) cudaEventDestroy(ctx->ev_side_fork);
    if (ctx->ev_side_join) cudaEventDestroy(ctx->ev_side_join);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    for (int c = 0; c < b2m::kNumCls; ++c)
        for (cudaEvent_t e : ctx->prof.ev[c]) cudaEventDestroy(e);
    for (auto& g : ctx->graphs) cudaGraphExecDestroy(g.second.exec);
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
    delete ctx;
    return B2M_OK;
}

extern "C" int32_t b2m_set_stream(b2m_ctx* h, void* stream) {
    Ctx* ctx = reinterpret_cast<Ctx*>(h);
    if (!ctx) return B2M_ERR_ARG;
    ctx->stream = reinterpret_cast<cudaStream_t>(stream);
    return B2M_OK;
}

extern "C" int32_t b2m_use_own_stream(b2m_ctx* h) {
    Ctx* ctx = reinterpret_cast<Ctx*>(h);
    if (!ctx) return B2M_ERR_ARG;
    ctx->stream = ctx->own_stream;
    return B2M_OK;
}

extern "C" int32_t b2m_profile(b2m_ctx* h, int32_t enable) {
    Ctx* ctx = reinterpret_cast<Ctx*>(h);
    if (!ctx) return B2M_ERR_ARG;
    B2M_CU(ctx, cudaStreamSynchronize(ctx->stream));
    ctx->prof.on = enable != 0;
    for (int c = 0; c < b2m::kNumCls; ++c) {
        ctx->prof.used[c] = 0;
        ctx->prof.work[c] = 0.0;
    }
    return B2M_OK;
}

extern "C" int32_t b2m_profile_read(b2m_ctx* h, int32_t cls, int64_t* launches, double* ms, double* work) {
    Ctx* ctx = reinterpret_cast<Ctx*>(h);
    if (!ctx || cls < 0 || cls >= b2m::kNumCls) return B2M_ERR_ARG;
    B2M_CU(ctx, cudaDeviceSynchronize());
    b2m::Prof& p = ctx->prof;
    double tot = 0.0;
    for (size_t i = 0; i + 1 < p.used[cls]; i += 2) {
        float t = 0.f;
        if (cudaEventElapsedTime(&t, p.ev[cls][i], p.ev[cls][i + 1]) == cudaSuccess) tot += t;
    }
    if (launches) *launches = (int64_t)(p.used[cls] / 2);
    if (ms) *ms = tot;
    if (work) *work = p.work[cls];
    return B2M_OK;
}

extern "C" int32_t b2m_use_graphs(b2m_ctx* h, int32_t enable) {
    Ctx* ctx = reinterpret_cast<Ctx*>(h);
    if (!ctx) return B2M_ERR_ARG;
    ctx->use_graphs = enable != 0;
    return B2M_OK;
}

extern "C" int32_t b2m_set_wait_limit(b2m_ctx* h, int64_t polls) {
    Ctx* ctx = reinterpret_cast<Ctx*>(h);
    if (!ctx) return B2M_ERR_ARG;
    b2m::CallLock lk(ctx);
    if (polls > 0xFFFFFFFFll) return b2m::fail(ctx, B2M_ERR_ARG, "wait limit above 2^32 - 1 polls");
    cudaSetDevice(ctx->device);
    // the limit is a kernel argument, so captured graphs that hold the old one are dropped
    B2M_CU(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->own_stream) B2M_CU(ctx, cudaStreamSynchronize(ctx->own_stream));
    for (auto& g : ctx->graphs) cudaGraphExecDestroy(g.second.exec);
    ctx->graphs.clear();
    ctx->wait_limit = polls < 0 ? -1 : polls;
    return B2M_OK;
}

// ------------------------------------------------------------------ resident matrices
extern "C" int32_t b2m_alloc(b2m_ctx* h, int64_t rows, int64_t cols, double** out, int64_t* LineWidth) {
    Ctx* ctx = reinterpret_cast<Ctx*>(h);
    if (!ctx || !out || !LineWidth) return B2M_ERR_ARG;
    *out = nullptr;
    *LineWidth = 0;
    if (rows < 0 || cols < 0) return b2m::fail(ctx, B2M_ERR_DIM, "negative dimension");
    // rows padded to 16 doubles (128 bytes): TMA-legal strides and coalesced rows, like the
    // library's own workspaces; at least one element so that an empty matrix has an address
    const int64_t ld = b2m::round_up(std::max<int64_t>(cols, 1), 16);
    cudaSetDevice(ctx->device);
    void* p = nullptr;
    if (cudaMalloc(&p, (size_t)(std::max<int64_t>(rows, 1) * ld * 8)) != cudaSuccess) {
        cudaGetLastError();
        return b2m::fail(ctx, B2M_ERR_ALLOC, "b2m_alloc: %lld x %lld doubles", (long long)rows, (long long)cols);
    }
    *out = static_cast<double*>(p);
    *LineWidth = ld * 8;
    return B2M_OK;
}

extern "C" int32_t b2m_free(b2m_ctx* h, double* p) {
    Ctx* ctx = reinterpret_cast<Ctx*>(h);
    if (!ctx) return B2M_ERR_ARG;
    if (!p) return B2M_OK;
    cudaSetDevice(ctx->device);
    B2M_CU(ctx, cudaStreamSynchronize(ctx->stream));  // queued work may still read it
    B2M_CU(ctx, cudaFree(p));
    return B2M_OK;
}

extern "C" int32_t b2m_upload(b2m_ctx* h, double* dst, int64_t dstLineWidth, const double* src, int64_t srcLineWidth,
                              int64_t rows, int64_t cols) {
    Ctx* ctx = reinterpret_cast<Ctx*>(h);
    if (!ctx || !dst || !src) return B2M_ERR_ARG;
    if (rows < 0 || cols < 0 || dstLineWidth < cols * 8 || srcLineWidth < cols * 8)
        return b2m::fail(ctx, B2M_ERR_DIM, "Line widths do not match");
    if (rows == 0 || cols == 0) return B2M_OK;
    b2m::CallLock lk(ctx);
    cudaSetDevice(ctx->device);
    B2M_CU(ctx, cudaMemcpy2DAsync(dst, dstLineWidth, src, srcLineWidth, cols * 8, rows, cudaMemcpyHostToDevice,
                                  ctx->stream));
    B2M_CU(ctx, cudaStreamSynchronize(ctx->stream));
    return B2M_OK;
}

extern "C" int32_t b2m_download(b2m_ctx* h, double* dst, int64_t dstLineWidth, const double* src,
                                int64_t srcLineWidth, int64_t rows, int64_t cols) {
    Ctx* ctx = reinterpret_cast<Ctx*>(h);
    if (!ctx || !dst || !src) return B2M_ERR_ARG;
    if (rows < 0 || cols < 0 || dstLineWidth < cols * 8 || srcLineWidth < cols * 8)
        return b2m::fail(ctx, B2M_ERR_DIM, "Line widths do not match");
    if (rows == 0 || cols == 0) return B2M_OK;
    b2m::CallLock lk(ctx);
    cudaSetDevice(ctx->device);
    B2M_CU(ctx, cudaMemcpy2DAsync(dst, dstLineWidth, src, srcLineWidth, cols * 8, rows, cudaMemcpyDeviceToHost,
                                  ctx->stream));
    B2M_CU(ctx, cudaStreamSynchronize(ctx->stream));
    return B2M_OK;
}

extern "C" int32_t b2m_set_progress(b2m_ctx* h, b2m_progress_fn fn, void* user) {
    Ctx* ctx = reinterpret_cast<Ctx*>(h);
    if (!ctx) return B2M_ERR_ARG;
    b2m::CallLock lk(ctx);
    ctx->progress = fn;
    ctx->progress_user = user;
    return B2M_OK;
}

extern "C" int32_t b2m_synchronize(b2m_ctx* h) {
    Ctx* ctx = reinterpret_cast<Ctx*>(h);
    if (!ctx) return B2M_ERR_ARG;
    B2M_CU(ctx, cudaStreamSynchronize(ctx->stream));
    return B2M_OK;
}

extern "C" const char* b2m_last_error(b2m_ctx* h) {
    Ctx* ctx = reinterpret_cast<Ctx*>(h);
    return ctx ? ctx->last_error.c_str() : "null context";
}

extern "C" int64_t b2m_kernel_launches(b2m_ctx* h) {
    Ctx* ctx = reinterpret_cast<Ctx*>(h);
    return ctx ? ctx->launches : -1;
}

extern "C" int32_t b2m_ctx_info(b2m_ctx* h, int32_t what, int64_t* value) {
    Ctx* ctx = reinterpret_cast<Ctx*>(h);
    if (!ctx || !value) return B2M_ERR_ARG;
    b2m::CallLock lk(ctx);
    switch (what) {
        case B2M_INFO_NUM_SMS: *value = ctx->num_sms; return B2M_OK;
        case B2M_INFO_SWEEP_CTAS: *value = ctx->sweep_ctas; return B2M_OK;
        case B2M_INFO_CHAIN_CLUSTERS: *value = ctx->chain_clusters; return B2M_OK;
        case B2M_INFO_CHAIN_PROBE: *value = ctx->chain_probe_why; return B2M_OK;
        case B2M_INFO_CHAIN_CLUSTERS4: *value = ctx->chain_clusters4; return B2M_OK;
        case B2M_INFO_BATCH_BIG_WARPS: {
            const auto it = ctx->batch_tunes.find(ctx->batch_plan_sig);
            *value = it != ctx->batch_tunes.end()       ? it->second.big_warps
                     : ctx->batch_tunes.empty() ? 0 : ctx->batch_tunes.begin()->second.big_warps;
            return B2M_OK;
        }
        default: return b2m::fail(ctx, B2M_ERR_ARG, "unknown info key %d", what);
    }
}

extern "C" const char* b2m_status_string(int32_t s) {
    switch (s) {
        case B2M_OK: return "ok";
        case B2M_SINGULAR: return "matrix is singular";
        case B2M_ERR_DIM: return "dimension error";
        case B2M_ERR_CUDA: return "CUDA error";
        case B2M_ERR_ALLOC: return "allocation failed";
        case B2M_ERR_TIMEOUT: return "bounded device wait timed out";
        case B2M_ERR_ARG: return "invalid argument";
        case B2M_ERR_NOCONV: return "refinement did not converge";
        case B2M_ERR_UNSUPPORTED: return "unsupported size or device";
        case B2M_ERR_FORMAT: return "not a saved matrix stream";
        default: return "unknown status";
    }
}
