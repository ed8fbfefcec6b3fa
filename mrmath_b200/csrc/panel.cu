// panel.cu -- partial-pivoting factorisation of one tall panel (the leaf of the LU recursion).
//
// One thread-block cluster of C <= 16 CTAs factors an m x w panel (w <= W) whose rows are held
// in registers: CTA `rank` owns panel rows [rank*R, rank*R + R), thread t of a CTA owns rows
// t, t + 256, t + 512, ...  Per column the CTAs exchange, by st.async pushes into every CTA's
// shared memory completing on that CTA's mbarrier, (a) their best pivot candidate with its full
// row and (b) the current diagonal row; each CTA then waits only on its own mbarrier and reads
// everything locally.  One __syncthreads and one one-way DSMEM latency per column -- no cluster
// barrier inside the loop.  Receive buffers, warp-winner rows and the mbarriers are double
// buffered by column parity, which the causal order of the pushes makes race-free: a CTA pushes
// column j+1 only after it has finished reading everything of column j.
//
// Pivot rule of the reference's leaf (LinAlgLU.pas:246-268): largest |a|, lowest row among
// equals, singular when the largest |a| is <= 10/MaxDouble; the column below the pivot is scaled
// by the reciprocal 1/pivot (MatrixScaleAndAdd computes x*Scale + Offset with Offset = 0).
#include <cooperative_groups.h>

#include <cfloat>

#include "common.cuh"
#include "kernels.cuh"

namespace cg = cooperative_groups;

namespace b2m {
namespace {

constexpr int kPT = 256;              // threads per CTA
constexpr int kPWarps = kPT / 32;
constexpr int kPMaxC = 16;            // largest cluster
constexpr int kPanelSmemMax = 200 * 1024;  // dynamic shared memory a panel CTA may use

template <typename T> __device__ __forceinline__ T sing_thresh();
template <> __device__ __forceinline__ double sing_thresh<double>() { return 10.0 / DBL_MAX; }
template <> __device__ __forceinline__ float sing_thresh<float>() { return 10.0f / FLT_MAX; }

template <typename T>
__device__ __forceinline__ bool better(T a2, int i2, T a1, int i1) {
    return i2 >= 0 && (i1 < 0 || a2 > a1 || (a2 == a1 && i2 < i1));
}

// Warp argmax with the reference's tie rule, exactly: |a| >= 0 orders like its bit pattern, so
// the maximum is found with integer reductions (high word, then low word), and the lowest row
// index among the lanes holding it wins.  Lanes without a candidate carry (0, -1).
__device__ __forceinline__ void warp_best(double& a, int& i) {
    const unsigned long long b = i >= 0 ? (unsigned long long)__double_as_longlong(a) : 0ull;
    const uint32_t hi = (uint32_t)(b >> 32), lo = (uint32_t)b;
    const uint32_t mhi = __reduce_max_sync(0xffffffffu, hi);
    const uint32_t m1 = __ballot_sync(0xffffffffu, hi == mhi && i >= 0);
    const uint32_t mlo = __reduce_max_sync(0xffffffffu, (m1 >> (threadIdx.x & 31)) & 1u ? lo : 0u);
    const bool top = i >= 0 && hi == mhi && lo == mlo;
    const uint32_t idx = __reduce_min_sync(0xffffffffu, top ? (uint32_t)i : 0xffffffffu);
    if (idx == 0xffffffffu) {
        a = 0.0;
        i = -1;
    } else {
        a = __longlong_as_double((long long)(((unsigned long long)mhi << 32) | mlo));
        i = (int)idx;
    }
}
__device__ __forceinline__ void warp_best(float& a, int& i) {
    const uint32_t key = i >= 0 ? __float_as_uint(a) : 0u;
    const uint32_t mk = __reduce_max_sync(0xffffffffu, key);
    const bool top = i >= 0 && key == mk;
    const uint32_t idx = __reduce_min_sync(0xffffffffu, top ? (uint32_t)i : 0xffffffffu);
    if (idx == 0xffffffffu) {
        a = 0.0f;
        i = -1;
    } else {
        a = __uint_as_float(mk);
        i = (int)idx;
    }
}

__device__ __forceinline__ uint4 pack_cand(double a, int i) {
    const unsigned long long b = __double_as_longlong(a);
    return make_uint4((uint32_t)b, (uint32_t)(b >> 32), (uint32_t)i, 0u);
}
__device__ __forceinline__ uint4 pack_cand(float a, int i) {
    return make_uint4(__float_as_uint(a), (uint32_t)i, 0u, 0u);
}
__device__ __forceinline__ void unpack_cand(const uint32_t* w, double& a, int& i) {
    a = __longlong_as_double(((unsigned long long)w[1] << 32) | w[0]);
    i = (int)w[2];
}
__device__ __forceinline__ void unpack_cand(const uint32_t* w, float& a, int& i) {
    a = __uint_as_float(w[0]);
    i = (int)w[1];
}

__device__ __forceinline__ void st_async_b32(uint32_t raddr, uint32_t v, uint32_t rbar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b32 [%0], %1, [%2];\n" ::"r"(raddr), "r"(v),
                 "r"(rbar)
                 : "memory");
}
__device__ __forceinline__ void st_async_b64(uint32_t raddr, unsigned long long v, uint32_t rbar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b64 [%0], %1, [%2];\n" ::"r"(raddr), "l"(v),
                 "r"(rbar)
                 : "memory");
}
__device__ __forceinline__ void st_async_elem(uint32_t raddr, double v, uint32_t rbar) {
    st_async_b64(raddr, (unsigned long long)__double_as_longlong(v), rbar);
}
__device__ __forceinline__ void st_async_elem(uint32_t raddr, float v, uint32_t rbar) {
    st_async_b32(raddr, __float_as_uint(v), rbar);
}

// The panel lives in shared memory column-major (S[c*RS + local row], RS odd): a column is a
// contiguous, conflict-free vector, and a row is one element per lane.
template <typename T, int W, int RPT>
__global__ void __launch_bounds__(kPT, 1)
    panel_push_kernel(T* P, int64_t ld, int m, int w, int R, int row_base, int col_base, int32_t* ipiv,
                      int32_t* status) {
    constexpr int RB = W * (int)sizeof(T);  // row bytes

    cg::cluster_group cluster = cg::this_cluster();
    const int C = (int)cluster.num_blocks();
    const int rank = (int)cluster.block_rank();

    extern __shared__ __align__(16) unsigned char panel_dyn[];
    T* S = reinterpret_cast<T*>(panel_dyn);
    const int RS = R | 1;

    __shared__ __align__(16) T rrow[2][kPMaxC][W];     // candidates' rows, by source CTA
    __shared__ __align__(16) T rdrow[2][W];            // the current diagonal row
    __shared__ __align__(16) uint32_t rcand[2][kPMaxC][4];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ T wabs[2][kPWarps];
    __shared__ int widx[2][kPWarps];

    if (status[kInfo] != 0) return;  // uniform over the cluster: written before this launch

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int lo = rank * R;
    const int hi = min(m, lo + R);
    const int nr = max(0, hi - lo);
    const uint32_t phase_bytes = (uint32_t)(C * (RB + 16) + RB);

    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_barrier_init();
    }
    // load this CTA's rows (row-major in global, column-major here), 16 loads in flight per thread
    {
        constexpr int B = 16;
        const int total = nr * W;
        for (int e0 = 0; e0 < total; e0 += B * kPT) {
            T v[B];
#pragma unroll
            for (int q = 0; q < B; ++q) {
                const int e = e0 + q * kPT + tid;
                const int rl = e / W, c = e - rl * W;
                v[q] = (e < total && c < w) ? P[(int64_t)(lo + rl) * ld + c] : T(0);
            }
#pragma unroll
            for (int q = 0; q < B; ++q) {
                const int e = e0 + q * kPT + tid;
                if (e < total) S[(e % W) * RS + e / W] = v[q];
            }
        }
    }
    cluster.sync();  // every mbarrier is initialised (and S is loaded) before the first push
    if (tid == 0) {
        mbar_arrive_expect_tx(&bar[0], phase_bytes);
        if (w > 1) mbar_arrive_expect_tx(&bar[1], phase_bytes);
    }

    // Columns are factored in blocks of BK: a block's columns live in registers (act), so each
    // column's scaling and rank-1 update touch registers only; the columns to the right of the
    // block receive one rank-BK update when the block is done.  Beyond the block, pushed rows are
    // therefore stale; the block's pivot rows get the missing triangular correction at the block
    // end (ublk), and every other row receives its own pending update with its own multipliers,
    // so each element sees exactly the sequence of rank-1 updates of the unblocked algorithm.
    constexpr int BK = 8;
    __shared__ __align__(16) T ublk[BK][W];
    int rowg[RPT];
    T act[RPT][BK];
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
        const int rl = tid + k * kPT;
        rowg[k] = rl < nr ? lo + rl : -1;
    }
    auto load_act = [&](const int jb) {
#pragma unroll
        for (int k = 0; k < RPT; ++k)
#pragma unroll
            for (int t = 0; t < BK; ++t)
                act[k][t] = (rowg[k] >= 0 && jb + t < W) ? S[(jb + t) * RS + tid + k * kPT] : T(0);
    };
    auto store_row = [&](const int k, const int jb) {
#pragma unroll
        for (int t = 0; t < BK; ++t)
            if (jb + t < w) S[(jb + t) * RS + tid + k * kPT] = act[k][t];
    };

    // CTA-reduce the candidates of column `col` and push them, with the winner's row and the
    // diagonal row `col`, to every CTA of the cluster (block columns are taken from registers)
    auto publish = [&](const int col, T ma, int mi, const int jb) {
        const int par = col & 1;
        warp_best(ma, mi);
#pragma unroll
        for (int k = 0; k < RPT; ++k)
            if (rowg[k] >= 0 && ((mi >= 0 && rowg[k] == mi) || rowg[k] == col)) store_row(k, jb);
        if (lane == 0) { wabs[par][warp] = ma; widx[par][warp] = mi; }
        __syncthreads();
        T a = lane < kPWarps ? wabs[par][lane] : T(0);
        int i = lane < kPWarps ? widx[par][lane] : -1;
        warp_best(a, i);
        const int wl = i >= 0 ? i - lo : 0;
        const bool own_diag = col >= lo && col < hi;
        for (int d = warp; d < C; d += kPWarps) {
            const uint32_t rb = map_rank(&bar[par], d);
            if (lane < W) {
                st_async_elem(map_rank(&rrow[par][rank][lane], d), S[lane * RS + wl], rb);
                if (own_diag) st_async_elem(map_rank(&rdrow[par][lane], d), S[lane * RS + (col - lo)], rb);
            }
            if (lane == 0) st_async16(map_rank(&rcand[par][rank][0], d), pack_cand(a, i), rb);
        }
        __syncthreads();  // rows read above are rewritten by the next column's interchange
    };

    load_act(0);
    {
        T ma = T(0);
        int mi = -1;
#pragma unroll
        for (int k = 0; k < RPT; ++k)
            if (rowg[k] >= 0 && fabs(act[k][0]) > ma) { ma = fabs(act[k][0]); mi = rowg[k]; }
        publish(0, ma, mi, 0);
    }
    bool stop = false;
    int jb = 0;
    for (; jb < w && !stop; jb += BK) {
#pragma unroll
        for (int t = 0; t < BK; ++t) {
            const int j = jb + t;
            if (j >= w) break;
            const int par = j & 1;
            bool ok = false;
            for (uint32_t it = 0; it < kSpinLimit; ++it)
                if (mbar_try_wait_cluster(&bar[par], (j >> 1) & 1)) { ok = true; break; }
            if (!ok) {
                atomicExch(&status[kTimeout], 201);
                stop = true;
                break;
            }
            if (tid == 0 && j + 2 < w) mbar_arrive_expect_tx(&bar[par], phase_bytes);
            // every warp derives the same pivot from the C candidates (lane c reads candidate c)
            T babs = T(0);
            int bidx = -1;
            if (lane < C) unpack_cand(&rcand[par][lane][0], babs, bidx);
            warp_best(babs, bidx);
            if (bidx < 0 || !(babs > sing_thresh<T>())) {
                if (rank == 0 && tid == 0) atomicExch(&status[kInfo], 1);
                stop = true;
                break;
            }
            const int bc = bidx / R;  // the CTA that owns the pivot row sent its row
            const T* u = &rrow[par][bc][0];
            const T* dr = &rdrow[par][0];
            const int p = bidx;
            if (rank == 0 && tid == 0) ipiv[col_base + j] = row_base + p;
            if (tid < W) ublk[t][tid] = u[tid];
            // the interchanged rows' columns outside the block: written lane-per-column by the
            // warp that owns each row (read only after the next barrier)
            if (j >= lo && j < hi && warp == ((j - lo) % kPT) >> 5 && lane < w && (lane < jb || lane >= jb + BK))
                S[lane * RS + (j - lo)] = u[lane];
            if (p != j && p >= lo && p < hi && warp == ((p - lo) % kPT) >> 5 && lane < w &&
                (lane < jb || lane >= jb + BK))
                S[lane * RS + (p - lo)] = dr[lane];
            const T rinv = T(1) / u[j];
            T mb = T(0);
            int mbi = -1;
#pragma unroll
            for (int k = 0; k < RPT; ++k) {
                const int r = rowg[k];
                if (r < 0) continue;
                const int rl = tid + k * kPT;
                // interchange: row j takes the pivot row, row p the old diagonal row (block
                // columns in registers, the rest in shared memory, written by the row's owner)
                if (r == j || r == p) {
                    const T* src = r == j ? u : dr;
#pragma unroll
                    for (int t2 = 0; t2 < BK; ++t2) act[k][t2] = src[jb + t2];
                }
                if (r > j) {
                    const T l = act[k][t] * rinv + T(0);
                    act[k][t] = l;
#pragma unroll
                    for (int t2 = t + 1; t2 < BK; ++t2) act[k][t2] = fma(-l, u[jb + t2], act[k][t2]);
                    if (t + 1 < BK && fabs(act[k][t + 1]) > mb) { mb = fabs(act[k][t + 1]); mbi = r; }
                }
            }
            if (j + 1 >= w) continue;
            if (t + 1 < BK) {
                publish(j + 1, mb, mbi, jb);
                continue;
            }
            // ---- block end: correct the block's pivot rows beyond the block (L11^{-1} U12), store
            // the block columns, rank-BK update of the columns to the right, load the next block
            __syncthreads();
            for (int c = jb + BK + tid; c < w; c += kPT) {
#pragma unroll
                for (int t1 = 1; t1 < BK; ++t1) {
                    T x = ublk[t1][c];
#pragma unroll
                    for (int t0 = 0; t0 < t1; ++t0) x = fma(-ublk[t1][jb + t0], ublk[t0][c], x);
                    ublk[t1][c] = x;
                }
            }
            __syncthreads();
#pragma unroll
            for (int k = 0; k < RPT; ++k) {
                const int r = rowg[k];
                if (r < 0) continue;
                const int rl = tid + k * kPT;
                store_row(k, jb);
                if (r > j) {
                    for (int c = jb + BK; c < w; ++c) {
                        T x = S[c * RS + rl];
#pragma unroll
                        for (int t2 = 0; t2 < BK; ++t2) x = fma(-act[k][t2], ublk[t2][c], x);
                        S[c * RS + rl] = x;
                    }
                } else if (r >= jb) {
                    for (int c = jb + BK; c < w; ++c) S[c * RS + rl] = ublk[r - jb][c];
                }
            }
            load_act(jb + BK);
            T ma = T(0);
            int mi = -1;
#pragma unroll
            for (int k = 0; k < RPT; ++k)
                if (rowg[k] > j && fabs(act[k][0]) > ma) { ma = fabs(act[k][0]); mi = rowg[k]; }
            publish(j + 1, ma, mi, jb + BK);
        }
    }
    if (!stop) {
        // the last block's columns are still in registers
        const int jl = ((w - 1) / BK) * BK;
#pragma unroll
        for (int k = 0; k < RPT; ++k)
            if (rowg[k] >= 0) store_row(k, jl);
    }
    __syncthreads();
    if (!stop) {
        for (int e = tid; e < nr * w; e += kPT) {
            const int rl = e / w, c = e - rl * w;
            P[(int64_t)(lo + rl) * ld + c] = S[c * RS + rl];
        }
    }
    cluster.sync();  // no CTA leaves while a push to it may still be in flight
}

template <typename T, int W, int RPT>
int32_t launch_push(Ctx* ctx, cudaStream_t st, int C, int R, T* P, int64_t ld, int m, int w, int row_base,
                    int col_base, int32_t* ipiv) {
    auto kern = panel_push_kernel<T, W, RPT>;
    const size_t smem = (size_t)W * (R | 1) * sizeof(T);
    std::atomic<int>& attr = device_flag((const void*)kern, 0, ctx->device);
    if (!attr.load()) {
        B2M_CU(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        B2M_CU(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kPanelSmemMax));
        attr.store(1);
    }
    // whether a cluster of C CTAs fits on this device: 1 yes, -1 no, 0 not asked yet
    std::atomic<int>& sched = device_flag((const void*)kern, 1 + C, ctx->device);
    cudaLaunchAttribute at[2];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    // the panel is the factorisation's critical path: when a look-ahead trailing update runs beside
    // it, its CTAs take free SMs ahead of the update's tiles
    at[1].id = cudaLaunchAttributePriority;
    at[1].val.priority = ctx->chain_priority;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(C, 1, 1);
    cfg.blockDim = dim3(kPT, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = 2;
    if (C > 8 && sched.load() == 0) {
        int clusters = 0;
        B2M_CU(ctx, cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg));
        sched.store(clusters > 0 ? 1 : -1);
    }
    if (C > 8 && sched.load() < 0)
        return fail(ctx, B2M_ERR_UNSUPPORTED, "panel cluster of %d CTAs cannot be scheduled", C);
    prof_begin(ctx, st, kClsPanel);
    B2M_CU(ctx, cudaLaunchKernelEx(&cfg, kern, P, ld, m, w, R, row_base, col_base, ipiv, ctx->d_status));
    prof_end(ctx, st, kClsPanel, 2.0 * m * w * sizeof(T));  // bytes: the panel read and written once
    B2M_LAUNCHED(ctx);
    return B2M_OK;
}

}  // namespace

// Tallest panel of width w: 16 CTAs x 256 threads x rows per thread (2 for w <= 32, 4 for w <= 16,
// 8 for w <= 8), the register budget of a row's block columns setting the rows per thread.
int panel_max_rows(bool fp64, int w) {
    if (fp64) return w <= 8 ? kPMaxC * kPT * 8 : (w <= 16 ? kPMaxC * kPT * 4 : kPMaxC * kPT * 2);
    return kPMaxC * kPT * 4;
}

template <typename T>
int32_t launch_panel(Ctx* ctx, cudaStream_t st, T* P, int64_t ld, int m, int w, int row_base, int col_base,
                     int32_t* ipiv) {
    if (w < 1 || w > 32 || m < w) return fail(ctx, B2M_ERR_DIM, "panel %d x %d", m, w);
    if constexpr (sizeof(T) == 8) {
        if (w > 16) {
            const int C = (int)ceil_div(m, kPT * 2);
            if (C > kPMaxC) return fail(ctx, B2M_ERR_UNSUPPORTED, "FP64 panel of %d rows needs width <= 16", m);
            return launch_push<T, 32, 2>(ctx, st, C, (int)ceil_div(m, C), P, ld, m, w, row_base, col_base, ipiv);
        }
        if (m > panel_max_rows(true, 16)) {  // very tall: 8 columns, 8 rows per thread
            const int C = (int)ceil_div(m, kPT * 8);
            if (w > 8 || C > kPMaxC)
                return fail(ctx, B2M_ERR_UNSUPPORTED, "FP64 panel of %d x %d is too tall", m, w);
            return launch_push<T, 8, 8>(ctx, st, C, (int)ceil_div(m, C), P, ld, m, w, row_base, col_base, ipiv);
        }
        const int C = (int)ceil_div(m, kPT * 4);
        if (C > kPMaxC) return fail(ctx, B2M_ERR_UNSUPPORTED, "FP64 panel of %d rows is too tall", m);
        return launch_push<T, 16, 4>(ctx, st, C, (int)ceil_div(m, C), P, ld, m, w, row_base, col_base, ipiv);
    } else {
        static_assert(sizeof(T) == 8, "the cluster panel is instantiated for FP64 only");
        return B2M_ERR_UNSUPPORTED;
    }
}

template int32_t launch_panel<double>(Ctx*, cudaStream_t, double*, int64_t, int, int, int, int, int32_t*);

}  // namespace b2m
