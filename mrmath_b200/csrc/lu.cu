// lu.cu -- partial-pivoting LU and the triangular solves built on it (FP64 plain form).
//
// Structure (a B200 re-design of InternalRecursiveMatrixLUDecompInPlace, LinAlgLU.pas:181-281):
//   * orders up to 512: the recursion splits the column range in two halves rounded to the
//     32-column leaf width (the reference halves exactly: mn div 2); larger orders: 256-column
//     outer panels with look-ahead, factored right-looking by leaves (lu_blocked below); the
//     leaves are factored by one thread-block cluster per panel with the panel resident in
//     distributed shared memory;
//   * a leaf's <= 32 row interchanges are applied at once to every other column of the matrix
//     (and to a row-permutation vector) by one swap launch, which replaces the reference's two
//     LUSwap calls per recursion level (:205, :237) -- the final matrix and pivot vector are the
//     same because each interchange is applied to every column exactly once, in order;
//   * A12 <- L11^{-1} A12 (LUBacksup :138-169) is a recursive triangular solve whose leaves run
//     a 32 x 32 register kernel and whose off-diagonal work goes through the DMMA GEMM;
//   * A22 -= A21 * A12 (MatrixMultEx ... doSub, :221) is the DMMA GEMM with the doSub epilogue.
// Pivot search follows the reference's leaf exactly: the largest |a| wins, the first (lowest
// row) among equals wins, a column whose largest |a| is <= 10/MaxDouble is singular (:246-268);
// the pivot column is scaled by the reciprocal 1/maxVal, as MatrixScaleAndAdd does.
#include <cooperative_groups.h>

#include <cfloat>

#include "common.cuh"
#include "kernels.cuh"

namespace cg = cooperative_groups;

namespace b2m {

template <typename T> __device__ __forceinline__ T singular_threshold();
template <> __device__ __forceinline__ double singular_threshold<double>() { return 10.0 / DBL_MAX; }
template <> __device__ __forceinline__ float singular_threshold<float>() { return 10.0f / FLT_MAX; }

// (a2,i2) beats (a1,i1): larger magnitude, or equal magnitude and lower row (first maximum wins)
template <typename T>
__device__ __forceinline__ bool piv_better(T a2, int i2, T a1, int i1) {
    return i2 >= 0 && (i1 < 0 || a2 > a1 || (a2 == a1 && i2 < i1));
}

template <typename T>
__device__ __forceinline__ void warp_argmax(T& a, int& i) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        T a2 = __shfl_xor_sync(0xffffffffu, a, o);
        int i2 = __shfl_xor_sync(0xffffffffu, i, o);
        if (piv_better(a2, i2, a, i)) { a = a2; i = i2; }
    }
}

constexpr int kPanelW = 32;  // largest leaf width

// ------------------------------------------------------------------------------------------
// Row interchanges of one leaf, applied to the columns [col_lo, col_hi) outside the leaf's own
// columns, to the permutation vector and (when given) to the outer panel's row map.  Warp 0 turns
// the <= 32 sequential swaps into a list of row moves.
// ------------------------------------------------------------------------------------------
constexpr int kSwapThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kSwapThreads)
    leaf_swap_kernel(T* A, int64_t ld, int col_lo, int col_hi, int c0, int w, const int32_t* ipiv, int32_t* perm,
                     int32_t* pmap, const int32_t* status) {
    __shared__ int src_main[kPanelW];
    __shared__ int mv_dst[2 * kPanelW], mv_src[2 * kPanelW];
    __shared__ int n_moves;
    if (status[kInfo] != 0) return;
    const int tid = threadIdx.x, lane = tid & 31;
    if (tid < 32) {
        if (lane < w) src_main[lane] = c0 + lane;
        __syncwarp();
        int my_pos = -1, my_src = -1, n_extra = 0;
        const int qv = lane < w ? ipiv[c0 + lane] : 0;  // one load per lane, not w dependent loads
        for (int j = 0; j < w; ++j) {
            const int q = __shfl_sync(0xffffffffu, qv, j);
            if (q < c0 + w) {
                if (lane == 0 && q != c0 + j) {
                    const int t = src_main[j];
                    src_main[j] = src_main[q - c0];
                    src_main[q - c0] = t;
                }
            } else {
                const unsigned hit = __ballot_sync(0xffffffffu, my_pos == q);
                int owner;
                if (hit) {
                    owner = __ffs(hit) - 1;
                } else {
                    owner = n_extra++;
                    if (lane == owner) { my_pos = q; my_src = q; }
                }
                if (lane == owner) {
                    const int t = src_main[j];
                    src_main[j] = my_src;
                    my_src = t;
                }
            }
            __syncwarp();
        }
        // compact the moves (rows whose content changes)
        const bool mv_main = lane < w && src_main[lane] != c0 + lane;
        const bool mv_extra = lane < n_extra && my_src != my_pos;
        const unsigned bm = __ballot_sync(0xffffffffu, mv_main);
        const unsigned be = __ballot_sync(0xffffffffu, mv_extra);
        const int below = (1u << lane) - 1u;
        if (mv_main) {
            const int k = __popc(bm & below);
            mv_dst[k] = c0 + lane;
            mv_src[k] = src_main[lane];
        }
        if (mv_extra) {
            const int k = __popc(bm) + __popc(be & below);
            mv_dst[k] = my_pos;
            mv_src[k] = my_src;
        }
        if (lane == 0) n_moves = __popc(bm) + __popc(be);
    }
    __syncthreads();
    const int nm = n_moves;
    if (nm == 0) return;
    const int gc = col_lo + blockIdx.x * kSwapThreads + tid;
    const int col = gc < c0 ? gc : gc + w;  // the leaf's own columns are skipped
    if (col < col_hi) {
        T v[2 * kPanelW];
#pragma unroll
        for (int k = 0; k < 2 * kPanelW; ++k)
            if (k < nm) v[k] = A[(int64_t)mv_src[k] * ld + col];
#pragma unroll
        for (int k = 0; k < 2 * kPanelW; ++k)
            if (k < nm) A[(int64_t)mv_dst[k] * ld + col] = v[k];
    }
    if ((perm || pmap) && blockIdx.x == 0) {
        int pv = 0, qv = 0;
        if (tid < nm) {
            if (perm) pv = perm[mv_src[tid]];
            if (pmap) qv = pmap[mv_src[tid]];
        }
        __syncthreads();
        if (tid < nm) {
            if (perm) perm[mv_dst[tid]] = pv;
            if (pmap) pmap[mv_dst[tid]] = qv;
        }
    }
}

// Inside an outer panel of the blocked FP64 LU, right-looking by leaves: after a leaf is factored,
// (1) leaf_swap_u12_kernel applies its interchanges to the panel's other columns and, for the
// panel columns right of the leaf, turns the leaf's rows into U12 = L11^-1 A12 (thread per column:
// the <= 32 values of the column in the leaf's rows after the interchanges, then the unit-lower
// forward substitution with contributions in ascending order, as trsm_small_kernel computes it);
// (2) panel_rank_update_kernel subtracts L21 U12 from the rest of the panel (rows below the leaf).  Both
// only touch the outer panel's columns; the other columns get the panel's net permutation and one
// K = 256 update per panel.
constexpr int kSuThreads = 64;  // columns per CTA of leaf_swap_u12_kernel
template <typename T>
__global__ void __launch_bounds__(kSuThreads)
    leaf_swap_u12_kernel(T* A, int64_t ld, int col_lo, int col_hi, int c0, int w, const int32_t* ipiv, int32_t* perm,
                         int32_t* pmap, const int32_t* status) {
    __shared__ int src_main[kPanelW];
    __shared__ int mv_dst[2 * kPanelW], mv_src[2 * kPanelW];
    __shared__ int n_moves, n_main;
    __shared__ T s_l[kPanelW][kPanelW + 1];  // L11 (strictly lower part), s_l[j][i] = L(c0 + j, c0 + i)
    if (status[kInfo] != 0) return;
    const int tid = threadIdx.x, lane = tid & 31;
    batched_copy<kSuThreads, kPanelW * kPanelW / kSuThreads, T>(tid, kPanelW * kPanelW,
        [&](int e) {
            const int j = e / kPanelW, i = e - j * kPanelW;
            return (i < j && j < w) ? A[(int64_t)(c0 + j) * ld + c0 + i] : T(0);
        },
        [&](int e, T v) { s_l[e / kPanelW][e % kPanelW] = v; });
    if (tid < 32) {
        // The interchanges composed into moves.  Lane i holds sm = the original row whose content
        // ends in row c0 + i; lane e < n_extra holds a row q outside the leaf's rows that an
        // interchange reached (my_pos) and the original row whose content ends there (my_src).
        // Each interchange swaps two of these entries through shuffles (one warp, no shared
        // memory round trip per interchange).
        int sm = c0 + lane;
        int my_pos = -1, my_src = -1, n_extra = 0;
        const int qv = lane < w ? ipiv[c0 + lane] : 0;
        for (int j = 0; j < w; ++j) {
            const int q = __shfl_sync(0xffffffffu, qv, j);
            const int a = __shfl_sync(0xffffffffu, sm, j);
            if (q < c0 + w) {
                const int qi = q - c0;
                const int b = __shfl_sync(0xffffffffu, sm, qi);
                if (lane == j) sm = b;
                else if (lane == qi) sm = a;
            } else {
                const unsigned hit = __ballot_sync(0xffffffffu, my_pos == q);
                int owner;
                if (hit) {
                    owner = __ffs(hit) - 1;
                } else {
                    owner = n_extra++;
                    if (lane == owner) { my_pos = q; my_src = q; }
                }
                const int b = __shfl_sync(0xffffffffu, my_src, owner);
                if (lane == j) sm = b;
                if (lane == owner) my_src = a;
            }
        }
        if (lane < w) src_main[lane] = sm;
        const bool mv_main = lane < w && sm != c0 + lane;
        const bool mv_extra = lane < n_extra && my_src != my_pos;
        const unsigned bm = __ballot_sync(0xffffffffu, mv_main);
        const unsigned be = __ballot_sync(0xffffffffu, mv_extra);
        const int below = (1u << lane) - 1u;
        if (mv_main) {
            const int k = __popc(bm & below);
            mv_dst[k] = c0 + lane;
            mv_src[k] = sm;
        }
        if (mv_extra) {
            const int k = __popc(bm) + __popc(be & below);
            mv_dst[k] = my_pos;
            mv_src[k] = my_src;
        }
        if (lane == 0) { n_moves = __popc(bm) + __popc(be); n_main = __popc(bm); }
    }
    __syncthreads();
    const int nm = n_moves;
    const int gc = col_lo + blockIdx.x * kSuThreads + tid;
    const int col = (gc < c0 || col_lo >= c0 + w) ? gc : gc + w;  // the leaf's own columns are skipped
    if (col < col_hi) {
        // every read of this column happens before its first write
        if (col > c0) {  // right of the leaf: the leaf's rows after the interchanges, then U12
            // the moves into the leaf's rows are covered by x; only the moves out of them (the
            // extra entries, after the n_main moves into the leaf's rows) need their own values
            const int nmain = n_main, nx = nm - n_main;
            T x[kPanelW], v[kPanelW];
#pragma unroll
            for (int j = 0; j < kPanelW; ++j) x[j] = j < w ? A[(int64_t)src_main[j] * ld + col] : T(0);
#pragma unroll
            for (int e = 0; e < kPanelW; ++e)
                if (e < nx) v[e] = A[(int64_t)mv_src[nmain + e] * ld + col];
#pragma unroll
            for (int e = 0; e < kPanelW; ++e)
                if (e < nx) A[(int64_t)mv_dst[nmain + e] * ld + col] = v[e];
#pragma unroll
            for (int i = 0; i < kPanelW - 1; ++i) {
#pragma unroll
                for (int j = i + 1; j < kPanelW; ++j) x[j] = fma(-s_l[j][i], x[i], x[j]);
            }
#pragma unroll
            for (int j = 0; j < kPanelW; ++j)
                if (j < w) A[(int64_t)(c0 + j) * ld + col] = x[j];
        } else {
            T v[2 * kPanelW];
#pragma unroll
            for (int k = 0; k < 2 * kPanelW; ++k)
                if (k < nm) v[k] = A[(int64_t)mv_src[k] * ld + col];
#pragma unroll
            for (int k = 0; k < 2 * kPanelW; ++k)
                if (k < nm) A[(int64_t)mv_dst[k] * ld + col] = v[k];
        }
    }
    if ((perm || pmap) && blockIdx.x == 0 && nm > 0) {
        int pv = 0, qv = 0;
        if (tid < nm) {
            if (perm) pv = perm[mv_src[tid]];
            if (pmap) qv = pmap[mv_src[tid]];
        }
        __syncthreads();
        if (tid < nm) {
            if (perm) perm[mv_dst[tid]] = pv;
            if (pmap) pmap[mv_dst[tid]] = qv;
        }
    }
}

// A[r][c] -= sum_{k < w} A[r][c0 + k] * A[c0 + k][c] for rows [r_lo, n) and columns [cl, ch): the
// leaf's rank-w update of the rest of its outer panel.  64 x 64 tiles, 4 x 4 per thread, the
// L21 and U12 slices staged in shared memory; the w products of each element are accumulated in
// ascending k and subtracted once (as the GEMM's doSub epilogue does).
constexpr int kRuT = 64;
__global__ void __launch_bounds__(256, 2) panel_rank_update_kernel(double* A, int64_t ld, int n, int r_lo, int cl, int ch,
                                                          int c0, int w, const int32_t* status) {
    __shared__ double s_a[kRuT][kPanelW + 1];  // L21 rows of the tile
    __shared__ __align__(16) double s_b[kPanelW][kRuT];  // U12 columns of the tile
    if (status[kInfo] != 0) return;
    const int t = threadIdx.x, tx = t & 15, ty = t >> 4;
    const int tiles_x = (ch - cl + kRuT - 1) / kRuT, tiles = tiles_x * ((n - r_lo + kRuT - 1) / kRuT);
    for (int tl = blockIdx.x; tl < tiles; tl += gridDim.x) {  // a grid smaller than the tiles loops
        const int r0 = r_lo + (tl / tiles_x) * kRuT, cb = cl + (tl % tiles_x) * kRuT;
        batched_copy<256, kRuT * kPanelW / 256, double>(t, kRuT * kPanelW,
            [&](int e) {
                const int rr = e >> 5, k = e & 31, row = r0 + rr;
                return (row < n && k < w) ? A[(int64_t)row * ld + c0 + k] : 0.0;
            },
            [&](int e, double v) { s_a[e >> 5][e & 31] = v; });
        batched_copy<256, kPanelW * kRuT / 256, double>(t, kPanelW * kRuT,
            [&](int e) {
                const int k = e / kRuT, col = cb + e % kRuT;
                return (k < w && col < ch) ? A[(int64_t)(c0 + k) * ld + col] : 0.0;
            },
            [&](int e, double v) { s_b[e / kRuT][e % kRuT] = v; });
        // the tile's own values, loaded while the slices arrive
        double c[4][4];
    #pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int row = r0 + 4 * ty + i;
    #pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int col = cb + 4 * tx + j;
                c[i][j] = (row < n && col < ch) ? A[(int64_t)row * ld + col] : 0.0;
            }
        }
        __syncthreads();
        double acc[4][4];
    #pragma unroll
        for (int i = 0; i < 4; ++i)
    #pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
    #pragma unroll 8
        for (int k = 0; k < kPanelW; ++k) {
            const double2 b01 = *reinterpret_cast<const double2*>(&s_b[k][4 * tx]);
            const double2 b23 = *reinterpret_cast<const double2*>(&s_b[k][4 * tx + 2]);
            const double bv[4] = {b01.x, b01.y, b23.x, b23.y};
    #pragma unroll
            for (int i = 0; i < 4; ++i) {
                const double av = s_a[4 * ty + i][k];
    #pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(av, bv[j], acc[i][j]);
            }
        }
    #pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int row = r0 + 4 * ty + i;
    #pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int col = cb + 4 * tx + j;
                if (row < n && col < ch) A[(int64_t)row * ld + col] = c[i][j] - acc[i][j];
            }
        }
        __syncthreads();  // the tile's slices are no longer read
    }
}

// U12 = L11^-1 A12 for one outer panel in a single launch: L11 unit lower (k <= 256 rows, at L with
// row stride ldl), the right-hand sides k x ncols at B.  A CTA owns 32 columns, held in shared
// memory for the whole solve; per 32-row block of L11 (staged in shared memory by cp.async, the
// next block column while the current one is used): warp 0 substitutes the block's diagonal
// triangle (lane = column; contributions in ascending order, as trsm_small_kernel computes them),
// then every warp subtracts the block's contribution from the rows below it (each element's 32
// products accumulated in ascending order and subtracted once).
constexpr int kTpK = 256;   // rows of the panel
constexpr int kTpC = 32;    // columns per CTA
constexpr int kTpSmem = (kTpK * kTpC + 2 * kTpK * kPanelW) * (int)sizeof(double);  // 192 KiB

__global__ void __launch_bounds__(256, 1) trsm_panel_kernel(const double* L, int64_t ldl, double* B, int64_t ldb,
                                                            int k, int ncols, const int32_t* status) {
    extern __shared__ __align__(16) double tp_dyn[];
    double* s_x = tp_dyn;                         // [kTpK][kTpC] this CTA's columns
    double* s_l = tp_dyn + kTpK * kTpC;           // [2][kTpK][kPanelW] block columns of L11 (rows 32 i ..)
    if (status[kInfo] != 0) return;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int cb = blockIdx.x * kTpC;
    const int nb = (int)ceil_div(k, kPanelW);
    // block column i of L11: rows [32 i, k), columns [32 i, 32 i + 32) -> buffer i & 1 (16-byte pieces)
    auto stage = [&](int i) {
        double* dst = s_l + (i & 1) * kTpK * kPanelW;
        const int r0 = kPanelW * i, rows = k - r0;
        for (int e = t; e < rows * (kPanelW / 2); e += 256) {
            const int rr = e / (kPanelW / 2), q2 = e - rr * (kPanelW / 2);
            const int col = r0 + 2 * q2;
            const double* src = L + (int64_t)(r0 + rr) * ldl + col;
            cp_async16(dst + rr * kPanelW + 2 * q2, src, col + 1 < k ? 16 : (col < k ? 8 : 0));
        }
        cp_async_commit();
    };
    stage(0);
    batched_copy<256, 8, double>(t, kTpK * kTpC,
        [&](int e) {
            const int r = e / kTpC, c = e - r * kTpC;
            return (r < k && cb + c < ncols) ? B[(int64_t)r * ldb + cb + c] : 0.0;
        },
        [&](int e, double v) { s_x[e] = v; });
    for (int i = 0; i < nb; ++i) {
        if (i + 1 < nb) {
            stage(i + 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const double* lb = s_l + (i & 1) * kTpK * kPanelW;  // lb[(r - 32 i) * 32 + q] = L[r][32 i + q]
        const int r0 = kPanelW * i, bw = min(kPanelW, k - r0);
        if (warp == 0) {
            double x[kPanelW];
#pragma unroll
            for (int j = 0; j < kPanelW; ++j) x[j] = s_x[(r0 + min(j, bw - 1)) * kTpC + lane];
#pragma unroll
            for (int q = 0; q < kPanelW - 1; ++q) {
#pragma unroll
                for (int j = q + 1; j < kPanelW; ++j)
                    if (j < bw) x[j] = fma(-lb[j * kPanelW + q], x[q], x[j]);
            }
#pragma unroll
            for (int j = 0; j < kPanelW; ++j)
                if (j < bw) s_x[(r0 + j) * kTpC + lane] = x[j];
        }
        __syncthreads();
        // rows below the block: thread (warp, lane) updates rows r0 + bw + warp + 8 m of column lane
        double xb[kPanelW];
#pragma unroll
        for (int q = 0; q < kPanelW; ++q) xb[q] = q < bw ? s_x[(r0 + q) * kTpC + lane] : 0.0;
        for (int r = r0 + bw + warp; r < k; r += 8) {
            const double* lr = lb + (r - r0) * kPanelW;
            double acc = 0.0;
#pragma unroll
            for (int q = 0; q < kPanelW; q += 2) {
                const double2 l2 = *reinterpret_cast<const double2*>(lr + q);
                acc = fma(l2.x, xb[q], acc);
                acc = fma(l2.y, xb[q + 1], acc);
            }
            s_x[r * kTpC + lane] -= acc;
        }
        __syncthreads();  // the buffer of block i is restaged for block i + 2
    }
    for (int e = t; e < kTpK * kTpC; e += 256) {
        const int r = e / kTpC, c = e - r * kTpC;
        if (r < k && cb + c < ncols) B[(int64_t)r * ldb + cb + c] = s_x[e];
    }
}

// The outer panel's net row permutation applied to the columns [col_begin, col_end) outside it:
// row i of the rows [oc0, n) receives what row pmap[i] held when the panel started.  CTA per 32
// columns; each CTA lists the moved rows (at most 2 x 256 for a 256-column panel; warp-aggregated
// appends) and loads all of their sources into registers before any write.
constexpr int kPpMax = 512;
__global__ void __launch_bounds__(256) panel_permute_f64_kernel(double* A, int64_t ld, int n, int oc0, int col_begin,
                                                                int col_end, const int32_t* pmap, int32_t* status) {
    __shared__ int s_dst[kPpMax], s_src[kPpMax], s_cnt;
    if (status[kInfo] != 0) return;
    const int t = threadIdx.x, lane = t & 31;
    if (t == 0) s_cnt = 0;
    __syncthreads();
    constexpr int kScan = 16;  // row-map entries per thread per pass, all loaded before use
    for (int p0 = oc0; p0 < n; p0 += 256 * kScan) {
        int src[kScan];
#pragma unroll
        for (int u = 0; u < kScan; ++u) {
            const int i = p0 + 256 * u + t;
            src[u] = i < n ? pmap[i] : i;
        }
#pragma unroll
        for (int u = 0; u < kScan; ++u) {
            const int i = p0 + 256 * u + t;
            const bool mv = src[u] != i;
            const unsigned bal = __ballot_sync(0xffffffffu, mv);
            if (!bal) continue;  // warp-uniform
            int base = 0;
            if (lane == 0) base = atomicAdd(&s_cnt, __popc(bal));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (mv) {
                const int k = base + __popc(bal & ((1u << lane) - 1u));
                if (k < kPpMax) { s_dst[k] = i; s_src[k] = src[u]; }
            }
        }
    }
    __syncthreads();
    const int cnt = s_cnt;
    if (cnt > kPpMax) {  // a 256-column panel moves at most 512 rows; anything else is an internal error
        if (t == 0) atomicExch(&status[kTimeout], 202);
        return;
    }
    const int col = col_begin + blockIdx.x * 32 + lane, rg = t >> 5;
    const bool ok = col < col_end;
    double x[kPpMax / 8];
#pragma unroll
    for (int q = 0; q < kPpMax / 8; ++q) {
        const int k = rg + 8 * q;
        x[q] = (ok && k < cnt) ? A[(int64_t)s_src[k] * ld + col] : 0.0;
    }
    __syncthreads();  // every source of this CTA's columns is read before any row is written
#pragma unroll
    for (int q = 0; q < kPpMax / 8; ++q) {
        const int k = rg + 8 * q;
        if (ok && k < cnt) A[(int64_t)s_dst[k] * ld + col] = x[q];
    }
}

// ------------------------------------------------------------------------------------------
// Small triangular solves (k <= 32) on a strip of columns.  One warp handles 4 columns; lane i
// holds row i of the triangle (registers) and x_i of each column; at step j the final x_j is
// broadcast with a shuffle and every later row subtracts its multiple, so the dependent chain is
// 32 shuffle+FMA steps.  Lower: unit diagonal, contributions in ascending j (LUBacksup and the
// forward sweep of MatrixLUBackSubst).  Upper: x_j = (b_j - sum) / U[j][j] with a true division
// (the backward sweep, LinAlgLU.pas:362-382), contributions in descending j.
// ------------------------------------------------------------------------------------------
constexpr int kTrsmThreads = 128;
constexpr int kTrsmCpw = 4;  // columns per warp

template <typename T>
__global__ void __launch_bounds__(kTrsmThreads)
    trsm_small_kernel(const T* L, int64_t ldl, T* B, int64_t ldb, int k, int ncols, int upper,
                      const int32_t* status) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int c0 = (blockIdx.x * (kTrsmThreads / 32) + warp) * kTrsmCpw;
    // all global loads first: the status word, this lane's row of the triangle, its x values
    const int32_t st = status ? status[kInfo] : 0;
    T lrow[kPanelW];
#pragma unroll
    for (int j = 0; j < kPanelW; ++j) lrow[j] = (lane < k && j < k) ? L[(int64_t)lane * ldl + j] : T(0);
    T x[kTrsmCpw];
#pragma unroll
    for (int q = 0; q < kTrsmCpw; ++q)
        x[q] = (lane < k && c0 + q < ncols) ? B[(int64_t)lane * ldb + c0 + q] : T(0);
    if (st != 0 || c0 >= ncols) return;
    if (!upper) {
#pragma unroll
        for (int j = 0; j < kPanelW - 1; ++j) {
            if (j >= k) break;
#pragma unroll
            for (int q = 0; q < kTrsmCpw; ++q) {
                const T xj = __shfl_sync(0xffffffffu, x[q], j);
                if (lane > j) x[q] = fma(-lrow[j], xj, x[q]);
            }
        }
    } else {
#pragma unroll
        for (int j = kPanelW - 1; j >= 0; --j) {
            if (j >= k) continue;
#pragma unroll
            for (int q = 0; q < kTrsmCpw; ++q) {
                if (lane == j) x[q] = x[q] / lrow[j];
                const T xj = __shfl_sync(0xffffffffu, x[q], j);
                if (lane < j) x[q] = fma(-lrow[j], xj, x[q]);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < kTrsmCpw; ++q)
        if (lane < k && c0 + q < ncols) B[(int64_t)lane * ldb + c0 + q] = x[q];
}

__global__ void iota_kernel(int32_t* v, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = (int32_t)i;
}

// X[i][:] = B[perm[i]][:]
__global__ void gather_rows_kernel(double* X, int64_t ldx, const double* B, int64_t ldb, const int32_t* perm,
                                   int64_t n, int64_t nrhs) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * nrhs) return;
    const int64_t i = e / nrhs, c = e - i * nrhs;
    X[i * ldx + c] = B[(int64_t)perm[i] * ldb + c];
}

// perm from a LAPACK-style ipiv: sequential interchanges, on a shared-memory copy when `in_smem`
// (n ints fit), else directly in perm (global memory; one dependent swap per step)
__global__ void perm_from_ipiv_kernel(const int32_t* ipiv, int n, int32_t* perm, int in_smem) {
    extern __shared__ int32_t pv_dyn[];
    int32_t* pv = in_smem ? pv_dyn : perm;
    for (int i = threadIdx.x; i < n; i += blockDim.x) pv[i] = i;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 0; i < n; ++i) {
            const int q = ipiv[i];
            if (q != i && q >= 0 && q < n) {
                const int t = pv[i];
                pv[i] = pv[q];
                pv[q] = t;
            }
        }
    }
    __syncthreads();
    if (in_smem)
        for (int i = threadIdx.x; i < n; i += blockDim.x) perm[i] = pv[i];
}

// det = (-1)^{#i: ipiv[i] != i} * U[0][0] * U[1][1] * ... in this order (MatrixDeterminant :467-476);
// the diagonal is staged through shared memory 1024 entries at a time (launch with 1024 threads)
constexpr int kDetChunk = 1024;
__global__ void __launch_bounds__(kDetChunk)
    determinant_kernel(const double* LU, int64_t ld, int n, const int32_t* ipiv, const int32_t* status, double* det) {
    __shared__ double dg[kDetChunk];
    __shared__ int flips;
    if (threadIdx.x == 0) flips = 0;
    __syncthreads();
    int local = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (ipiv[i] != i) local++;
    atomicAdd(&flips, local);
    __syncthreads();
    double r = (flips & 1) ? -1.0 : 1.0;  // thread 0's running product
    for (int c0 = 0; c0 < n; c0 += kDetChunk) {
        const int i = c0 + (int)threadIdx.x;
        if (i < n) dg[threadIdx.x] = LU[(int64_t)i * ld + i];
        __syncthreads();
        if (threadIdx.x == 0) {
            const int cnt = min(kDetChunk, n - c0);
            for (int k = 0; k < cnt; ++k) r = r * dg[k];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *det = status[kInfo] != 0 ? 0.0 : r;
}

// ------------------------------------------------------------------------------------------
// host drivers
// ------------------------------------------------------------------------------------------
namespace {

int64_t split_cols(int64_t w) { return round_up((w + 1) / 2, kPanelW); }

void CUDART_CB progress_trampoline(void* p) {
    const ProgressNote* note = static_cast<const ProgressNote*>(p);
    if (note->fn) note->fn(note->percent, note->user);
}

// the leaf's interchanges on columns [col_lo, col_hi) (which contain the leaf's own columns)
template <typename T>
int32_t launch_swaps_range(Ctx* ctx, cudaStream_t st, T* A, int64_t ld, int col_lo, int col_hi, int c0, int w,
                           const int32_t* ipiv, int32_t* perm, int32_t* pmap) {
    const int other = col_hi - col_lo - w;
    const int blocks = std::max(1, (int)ceil_div(other, kSwapThreads));
    prof_begin(ctx, st, kClsSwap);
    leaf_swap_kernel<T><<<blocks, kSwapThreads, 0, st>>>(A, ld, col_lo, col_hi, c0, w, ipiv, perm, pmap,
                                                         ctx->d_status);
    prof_end(ctx, st, kClsSwap, 4.0 * w * other * sizeof(T));  // <= 2w rows read + written
    B2M_LAUNCHED(ctx);
    return B2M_OK;
}

template <typename T>
int32_t launch_swaps_impl(Ctx* ctx, cudaStream_t st, T* A, int64_t ld, int ncols, int c0, int w, const int32_t* ipiv,
                     int32_t* perm) {
    return launch_swaps_range<T>(ctx, st, A, ld, 0, ncols, c0, w, ipiv, perm, nullptr);
}

template <typename T>
int32_t launch_trsm_small_impl(Ctx* ctx, cudaStream_t st, const T* L, int64_t ldl, T* B, int64_t ldb, int k, int ncols,
                          bool upper) {
    if (k <= 0 || ncols <= 0) return B2M_OK;
    const int blocks = (int)ceil_div(ncols, (kTrsmThreads / 32) * kTrsmCpw);
    prof_begin(ctx, st, kClsTrsm);
    trsm_small_kernel<T><<<blocks, kTrsmThreads, 0, st>>>(L, ldl, B, ldb, k, ncols, upper ? 1 : 0, ctx->d_status);
    prof_end(ctx, st, kClsTrsm, (double)sizeof(T) * (k * k + 2.0 * k * ncols));  // bytes
    B2M_LAUNCHED(ctx);
    return B2M_OK;
}

// Triangular operand description for the recursive solves: the triangle T lives in the
// row-major array (Abase, lda, an n x n extent) at diagonal offset r0; the right-hand sides are
// rows [br0, br0+k) and columns [bc0, bc0+ncols) of (Bbase, ldb) whose map extent is bn x bcols.
struct TriSolve {
    const double* A;
    int64_t lda, n;
    double* B;
    int64_t ldb, bn, bcols, bc0, ncols;
};

int32_t trsm_lower_rec(Ctx* ctx, cudaStream_t st, const TriSolve& t, int64_t r0, int64_t br0, int64_t k) {
    if (k <= kPanelW)
        return launch_trsm_small_impl<double>(ctx, st, t.A + r0 * t.lda + r0, t.lda, t.B + br0 * t.ldb + t.bc0, t.ldb,
                                         (int)k, (int)t.ncols, false);
    const int64_t k1 = split_cols(k), k2 = k - k1;
    B2M_TRY(trsm_lower_rec(ctx, st, t, r0, br0, k1));
    DOperand a{t.A, t.lda, t.n, t.n, r0 + k1, r0, true};
    DOperand b{t.B, t.ldb, t.bn, t.bcols, br0, t.bc0, false};
    B2M_TRY(dgemm_tiled(ctx, st, a, b, t.B + (br0 + k1) * t.ldb + t.bc0, t.ldb, k2, t.ncols, k1, B2M_DO_SUB, true));
    return trsm_lower_rec(ctx, st, t, r0 + k1, br0 + k1, k2);
}

int32_t trsm_upper_rec(Ctx* ctx, cudaStream_t st, const TriSolve& t, int64_t r0, int64_t br0, int64_t k) {
    if (k <= kPanelW)
        return launch_trsm_small_impl<double>(ctx, st, t.A + r0 * t.lda + r0, t.lda, t.B + br0 * t.ldb + t.bc0, t.ldb,
                                         (int)k, (int)t.ncols, true);
    const int64_t k1 = split_cols(k), k2 = k - k1;
    B2M_TRY(trsm_upper_rec(ctx, st, t, r0 + k1, br0 + k1, k2));
    DOperand a{t.A, t.lda, t.n, t.n, r0, r0 + k1, true};
    DOperand b{t.B, t.ldb, t.bn, t.bcols, br0 + k1, t.bc0, false};
    B2M_TRY(dgemm_tiled(ctx, st, a, b, t.B + br0 * t.ldb + t.bc0, t.ldb, k1, t.ncols, k2, B2M_DO_SUB, true));
    return trsm_upper_rec(ctx, st, t, r0, br0, k1);
}

// where a leaf's interchanges go: the columns [col_lo, col_hi) (the whole matrix, or one outer
// panel whose other columns are permuted once per panel through the row map pmap)
struct SwapScope {
    int64_t col_lo, col_hi;
    int32_t* pmap;
};

// factor columns [c0, c0+width), rows [c0, n); leaves of at most `leaf` columns
int32_t lu_rec(Ctx* ctx, cudaStream_t st, double* A, int64_t ld, int64_t n, int64_t c0, int64_t width,
               int32_t* ipiv, int32_t* perm, int64_t leaf, const SwapScope& sc) {
    if (width <= leaf) {
        B2M_TRY(launch_panel<double>(ctx, st, A + c0 * ld + c0, ld, (int)(n - c0), (int)width, (int)c0, (int)c0,
                                     ipiv));
        B2M_TRY(launch_swaps_range<double>(ctx, st, A, ld, (int)sc.col_lo, (int)sc.col_hi, (int)c0, (int)width, ipiv,
                                           perm, sc.pmap));
        if (ctx->progress && ctx->progress_notes.size() < ctx->progress_notes.capacity()) {
            // TLinEquProgress: columns factored * 100 div n, queued behind this panel
            ctx->progress_notes.push_back(
                ProgressNote{ctx->progress, ctx->progress_user, (int32_t)((c0 + width) * 100 / n)});
            B2M_CU(ctx, cudaLaunchHostFunc(st, progress_trampoline, &ctx->progress_notes.back()));
        }
        return B2M_OK;
    }
    // splits on multiples of 16 above the leaf level keep the Schur GEMMs' K on whole TMA k-tiles
    // (8-column leaves then meet only in their own narrow K = 8 updates)
    const int64_t step = width > 16 ? std::max<int64_t>(leaf, 16) : leaf;
    const int64_t nleft = round_up((width + 1) / 2, step), nright = width - nleft;
    B2M_TRY(lu_rec(ctx, st, A, ld, n, c0, nleft, ipiv, perm, leaf, sc));
    // A12 <- L11^{-1} A12
    TriSolve t{A, ld, n, A, ld, n, n, c0 + nleft, nright};
    B2M_TRY(trsm_lower_rec(ctx, st, t, c0, c0, nleft));
    // A22 -= A21 * A12
    const int64_t r1 = c0 + nleft;
    DOperand a{A, ld, n, n, r1, c0, true};
    DOperand b{A, ld, n, n, c0, r1, false};
    B2M_TRY(dgemm_tiled(ctx, st, a, b, A + r1 * ld + r1, ld, n - r1, nright, nleft, B2M_DO_SUB, true));
    return lu_rec(ctx, st, A, ld, n, r1, nright, ipiv, perm, leaf, sc);
}

constexpr int64_t kOuterNB = 256;  // outer panel width of the blocked FP64 LU
static_assert(kOuterNB == kTpK, "the panel triangular solve holds one outer panel's rows");

// Blocked right-looking LU with look-ahead (orders n > 2 kOuterNB).  Per outer panel of 256
// columns: (1) the panel is factored right-looking by leaves, each leaf's interchanges kept inside
// the panel (and recorded in the row map pmap), its U12 formed by the same launch and its rank-w
// update applied to the rest of the panel (leaf_swap_u12_kernel, panel_rank_update_kernel); (2) the
// panel's net permutation is applied to the next panel's columns on this stream, and to every
// further column right of the panel and the factored columns left of it on the side stream;
// (3) U12 = L11^-1 A12 (trsm_panel_kernel, one launch) and A22 -= A21 U12 for the next panel's
// 256 columns on this stream;
// (4) the same for every further column on the side stream, where it overlaps the next panel's
// factorisation (which reads and writes only the next panel's columns) and is joined before the
// next step's permutation moves rows under it.  The row map alternates between two buffers by panel
// parity, because the side stream may still read one panel's map while the next panel fills its own.
// Every interchange reaches every column exactly once and in order, so the factors and the pivot
// vector are those of the unblocked recursion.
// part 0 issues the first outer panel's leaves only, part 1 everything after them (two graphs: the
// device factors the first panel while the host submits the second).
int32_t lu_blocked(Ctx* ctx, cudaStream_t q, double* A, int64_t ld, int64_t n, int32_t* ipiv, int32_t* perm,
                   int32_t* pmap2, int64_t leaf, int part) {
    cudaStream_t q2 = ctx->side_stream;
    bool side_busy = false;
    auto join = [&]() -> int32_t {
        if (!side_busy) return B2M_OK;
        B2M_CU(ctx, cudaEventRecord(ctx->ev_side_join, q2));
        B2M_CU(ctx, cudaStreamWaitEvent(q, ctx->ev_side_join, 0));
        side_busy = false;
        return B2M_OK;
    };
    auto fork = [&]() -> int32_t {
        B2M_CU(ctx, cudaEventRecord(ctx->ev_side_fork, q));
        B2M_CU(ctx, cudaStreamWaitEvent(q2, ctx->ev_side_fork, 0));
        side_busy = true;
        return B2M_OK;
    };
    const int64_t pm_ld = round_up(n, 64);
    PriorityScope hi(ctx, true);  // this stream's launches are the critical path (see launch_k)
    std::atomic<int>& attr = device_flag((const void*)trsm_panel_kernel, 0, ctx->device);
    if (!attr.load()) {
        B2M_CU(ctx, cudaFuncSetAttribute(trsm_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTpSmem));
        attr.store(1);
    }
    for (int64_t k0 = 0; k0 < n; k0 += kOuterNB) {
        const int64_t w = std::min(kOuterNB, n - k0), k1 = k0 + w;
        int32_t* pmap = pmap2 + ((k0 / kOuterNB) & 1) * pm_ld;
        const bool leaves = (part == 0) == (k0 == 0);
        if (leaves) {
            B2M_CU(ctx, launch_k(ctx, iota_kernel, dim3((unsigned)ceil_div(n, 256)), dim3(256), 0, q, pmap, n));
            B2M_LAUNCHED(ctx);
        }
        // The panel, right-looking by leaves.  The critical path, on this stream: a leaf's panel
        // kernel, then its interchanges, U12 and rank-w update on the next leaf's columns only; the
        // same for the other columns of the outer panel (the factored ones left of the leaf get the
        // interchanges only) runs on the leaf stream, under the next leaf's panel kernel, and is
        // waited for before that leaf's own updates touch those columns.  Column groups are
        // disjoint between the two streams, and every column sees the leaves' interchanges and
        // updates in leaf order, so the factors are those of the single-stream order.
        cudaStream_t ql = ctx->leaf_stream;
        bool leaf_busy = false;
        auto swap_u12 = [&](cudaStream_t qs, int64_t c0, int64_t wl, int64_t lo, int64_t hi, bool maps) -> int32_t {
            const int64_t cols = std::max<int64_t>(0, (lo >= c0 + wl || hi <= c0) ? hi - lo : hi - lo - wl);
            if (cols == 0 && !maps) return B2M_OK;  // (the maps' update runs even without columns)
            prof_begin(ctx, qs, kClsSwap);
            B2M_CU(ctx, launch_k(ctx, leaf_swap_u12_kernel<double>,
                                 dim3((unsigned)std::max<int64_t>(1, ceil_div(cols, kSuThreads))),
                                 dim3(kSuThreads), 0, qs, A, ld, (int)lo, (int)hi, (int)c0, (int)wl, ipiv,
                                 maps ? perm : (int32_t*)nullptr, maps ? pmap : (int32_t*)nullptr,
                                 (const int32_t*)ctx->d_status));
            prof_end(ctx, qs, kClsSwap, 16.0 * wl * (double)cols);
            B2M_LAUNCHED(ctx);
            return B2M_OK;
        };
        auto rank_update = [&](cudaStream_t qs, int64_t c0, int64_t wl, int64_t cl, int64_t ch, int max_ctas) -> int32_t {
            const int64_t rl = c0 + wl;
            if (ch <= cl || rl >= n) return B2M_OK;
            const int64_t tiles = ceil_div(ch - cl, kRuT) * ceil_div(n - rl, kRuT);
            prof_begin(ctx, qs, kClsGemm);
            B2M_CU(ctx, launch_k(ctx, panel_rank_update_kernel, dim3((unsigned)std::min<int64_t>(tiles, max_ctas)),
                                 dim3(256), 0, qs, A, ld, (int)n, (int)rl, (int)cl, (int)ch, (int)c0, (int)wl,
                                 (const int32_t*)ctx->d_status));
            prof_end(ctx, qs, kClsGemm, 2.0 * (double)(n - rl) * (double)(ch - cl) * (double)wl);  // flops
            B2M_LAUNCHED(ctx);
            return B2M_OK;
        };
        for (int64_t c0 = k0; leaves && c0 < k1; c0 += leaf) {
            const int64_t wl = std::min(leaf, k1 - c0);
            B2M_TRY(launch_panel<double>(ctx, q, A + c0 * ld + c0, ld, (int)(n - c0), (int)wl, (int)c0, (int)c0, ipiv));
            const int64_t rl = c0 + wl, nx = std::min(rl + leaf, k1);  // the next leaf: columns [rl, nx)
            B2M_CU(ctx, cudaEventRecord(ctx->ev_leaf_panel, q));
            if (leaf_busy) {  // the previous leaf's updates of [rl, k1) are done
                B2M_CU(ctx, cudaStreamWaitEvent(q, ctx->ev_leaf_side, 0));
                leaf_busy = false;
            }
            B2M_TRY(swap_u12(q, c0, wl, rl, nx, true));
            B2M_TRY(rank_update(q, c0, wl, rl, nx, 1 << 30));
            if (nx < k1 || c0 > k0) {
                PriorityScope side(ctx, false);
                B2M_CU(ctx, cudaStreamWaitEvent(ql, ctx->ev_leaf_panel, 0));
                B2M_TRY(swap_u12(ql, c0, wl, nx, k1, false));
                B2M_TRY(swap_u12(ql, c0, wl, k0, c0, false));
                B2M_TRY(rank_update(ql, c0, wl, nx, k1, 64));
                B2M_CU(ctx, cudaEventRecord(ctx->ev_leaf_side, ql));
                leaf_busy = true;
            }
            if (ctx->progress && ctx->progress_notes.size() < ctx->progress_notes.capacity()) {
                ctx->progress_notes.push_back(
                    ProgressNote{ctx->progress, ctx->progress_user, (int32_t)((c0 + wl) * 100 / n)});
                B2M_CU(ctx, cudaLaunchHostFunc(q, progress_trampoline, &ctx->progress_notes.back()));
            }
        }
        if (leaf_busy) B2M_CU(ctx, cudaStreamWaitEvent(q, ctx->ev_leaf_side, 0));
        if (part == 0) return B2M_OK;
        B2M_TRY(join());  // the previous panel's wide update is done before rows move under it
        auto permute = [&](cudaStream_t qs, int64_t c_begin, int64_t c_end) -> int32_t {
            if (c_end <= c_begin) return B2M_OK;
            prof_begin(ctx, qs, kClsSwap);
            B2M_CU(ctx, launch_k(ctx, panel_permute_f64_kernel, dim3((unsigned)ceil_div(c_end - c_begin, 32)), dim3(256), 0,
                                 qs, A, ld, (int)n, (int)k0, (int)c_begin, (int)c_end, (const int32_t*)pmap,
                                 ctx->d_status));
            prof_end(ctx, qs, kClsSwap, 2.0 * 8.0 * 2 * w * (double)(c_end - c_begin));  // <= 2w rows moved
            B2M_LAUNCHED(ctx);
            return B2M_OK;
        };
        const int64_t rest = n - k1, nw = std::min(kOuterNB, std::max<int64_t>(rest, 0));
        // only the next panel's columns are permuted on this stream; the other columns right of
        // the panel and the factored columns left of it on the side stream, ahead of their update
        B2M_TRY(permute(q, k1, k1 + nw));
        if (k0 > 0 || rest > nw) {
            B2M_TRY(fork());
            PriorityScope side(ctx, false);
            B2M_TRY(permute(q2, k1 + nw, n));
            B2M_TRY(permute(q2, 0, k0));
        }
        if (k1 >= n) break;
        auto update = [&](cudaStream_t qs, int64_t cs, int64_t nc) -> int32_t {
            prof_begin(ctx, qs, kClsTrsm);
            B2M_CU(ctx, launch_k(ctx, trsm_panel_kernel, dim3((unsigned)ceil_div(nc, kTpC)), dim3(256), (size_t)kTpSmem,
                                 qs, (const double*)(A + k0 * ld + k0), ld, A + k0 * ld + cs, ld, (int)w, (int)nc,
                                 (const int32_t*)ctx->d_status));
            prof_end(ctx, qs, kClsTrsm, 8.0 * (w * (double)w / 2 + 2.0 * w * (double)nc));  // bytes
            B2M_LAUNCHED(ctx);
            DOperand a{A, ld, n, n, k1, k0, true};
            DOperand b{A, ld, n, n, k0, cs, false};
            return dgemm_tiled(ctx, qs, a, b, A + k1 * ld + cs, ld, n - k1, nc, w, B2M_DO_SUB, true);
        };
        if (rest > nw) {
            PriorityScope side(ctx, false);
            B2M_TRY(update(q2, k1 + nw, rest - nw));
        }
        B2M_TRY(update(q, k1, nw));
    }
    return join();
}


}  // namespace

// the low-priority side stream (and its fork/join events) of this context, created on first use
int32_t ensure_side_stream(Ctx* ctx) {
    if (ctx->side_stream && ctx->leaf_stream) return B2M_OK;
    int least = 0, greatest = 0;
    B2M_CU(ctx, cudaDeviceGetStreamPriorityRange(&least, &greatest));
    if (!ctx->side_stream) {
        B2M_CU(ctx, cudaStreamCreateWithPriority(&ctx->side_stream, cudaStreamNonBlocking, least));
        B2M_CU(ctx, cudaEventCreateWithFlags(&ctx->ev_side_fork, cudaEventDisableTiming));
        B2M_CU(ctx, cudaEventCreateWithFlags(&ctx->ev_side_join, cudaEventDisableTiming));
    }
    // the FP64 LU's in-panel look-ahead: the stream runs at the critical path's priority, since the
    // leaf after next waits for it
    B2M_CU(ctx, cudaStreamCreateWithPriority(&ctx->leaf_stream, cudaStreamNonBlocking, greatest));
    B2M_CU(ctx, cudaEventCreateWithFlags(&ctx->ev_leaf_panel, cudaEventDisableTiming));
    B2M_CU(ctx, cudaEventCreateWithFlags(&ctx->ev_leaf_side, cudaEventDisableTiming));
    ctx->chain_priority = greatest;
    return B2M_OK;
}

template <typename T>
int32_t launch_swaps(Ctx* ctx, cudaStream_t st, T* A, int64_t ld, int ncols, int c0, int w, const int32_t* ipiv,
                     int32_t* perm) {
    return launch_swaps_impl<T>(ctx, st, A, ld, ncols, c0, w, ipiv, perm);
}
template <typename T>
int32_t launch_trsm_small(Ctx* ctx, cudaStream_t st, const T* L, int64_t ldl, T* B, int64_t ldb, int k, int ncols,
                          bool upper) {
    return launch_trsm_small_impl<T>(ctx, st, L, ldl, B, ldb, k, ncols, upper);
}
template int32_t launch_swaps<float>(Ctx*, cudaStream_t, float*, int64_t, int, int, int, const int32_t*, int32_t*);
template int32_t launch_swaps<double>(Ctx*, cudaStream_t, double*, int64_t, int, int, int, const int32_t*, int32_t*);
template int32_t launch_trsm_small<float>(Ctx*, cudaStream_t, const float*, int64_t, float*, int64_t, int, int, bool);
template int32_t launch_trsm_small<double>(Ctx*, cudaStream_t, const double*, int64_t, double*, int64_t, int, int,
                                           bool);

int32_t lu_factor_f64(Ctx* ctx, cudaStream_t st, double* A, int64_t ld, int64_t n, int32_t* ipiv, int32_t* perm) {
    if (n <= 0) return B2M_OK;
    if ((ld & 1) || !aligned16(A)) return fail(ctx, B2M_ERR_DIM, "lu_factor_f64: ld must be even, A 16-byte aligned");
    if (n > (1 << 30)) return fail(ctx, B2M_ERR_UNSUPPORTED, "n too large");
    // the leaf width shrinks as the first panel grows (the cluster holds a whole panel on chip)
    const int64_t leaf = n <= panel_max_rows(true, 32) ? 32 : (n <= panel_max_rows(true, 16) ? 16 : 8);
    if (n > panel_max_rows(true, 8))
        return fail(ctx, B2M_ERR_UNSUPPORTED, "FP64 LU supports n <= %d", panel_max_rows(true, 8));
    if (ctx->progress) {
        // the notes are the host functions' payloads: wait until the previous call's have run, then
        // reserve one per leaf so that none moves while queued
        B2M_CU(ctx, cudaStreamSynchronize(st));
        ctx->progress_notes.clear();
        ctx->progress_notes.reserve((size_t)(n / 8 + 2));
    }
    // orders above 2 outer panels take the blocked look-ahead driver (row maps in a workspace); smaller
    // ones (and every call of the allocation-free entry point, n <= 512) the plain recursion
    const bool blocked = n > 2 * kOuterNB;
    int32_t* pmap2 = nullptr;
    if (blocked) {
        void* p = nullptr;
        B2M_TRY(ws_get(ctx, kWsPmap, (size_t)(2 * round_up(n, 64)) * sizeof(int32_t), &p));
        pmap2 = static_cast<int32_t*>(p);
        B2M_TRY(ensure_side_stream(ctx));
    }
    const GraphKey key{1, A, ipiv, perm, ctx->d_status, ld, n, 0, 0};
    const GraphKey key1{1, A, ipiv, perm, ctx->d_status, ld, n, 0, 1};
    B2M_TRY(run_graph(ctx, st, key, [&](cudaStream_t s) -> int32_t {
        if (perm) {
            iota_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, s>>>(perm, n);
            B2M_LAUNCHED(ctx);
        }
        if (blocked) return lu_blocked(ctx, s, A, ld, n, ipiv, perm, pmap2, leaf, 0);
        return lu_rec(ctx, s, A, ld, n, 0, n, ipiv, perm, leaf, SwapScope{0, n, nullptr});
    }));
    if (!blocked) return B2M_OK;
    return run_graph(ctx, st, key1, [&](cudaStream_t s) -> int32_t {
        return lu_blocked(ctx, s, A, ld, n, ipiv, perm, pmap2, leaf, 1);
    });
}

int32_t lu_solve_f64(Ctx* ctx, cudaStream_t st, const double* LU, int64_t ld, int64_t n, const int32_t* perm,
                     double* B, int64_t ldb, int64_t nrhs, double* tmp) {
    if (n <= 0 || nrhs <= 0) return B2M_OK;
    if ((ldb & 1) || !aligned16(B)) return fail(ctx, B2M_ERR_DIM, "lu_solve_f64: ldb must be even");
    // X = P B
    double* X = tmp;
    if (!X) {
        void* w = nullptr;
        B2M_TRY(ws_get(ctx, kWsE, (size_t)(n * ldb * sizeof(double)), &w));
        X = static_cast<double*>(w);
    }
    const GraphKey key{2, LU, perm, B, X, ld, n, ldb, nrhs};
    return run_graph(ctx, st, key, [&](cudaStream_t s) -> int32_t {
        B2M_CU(ctx, cudaMemcpy2DAsync(X, ldb * 8, B, ldb * 8, nrhs * 8, n, cudaMemcpyDeviceToDevice, s));
        gather_rows_kernel<<<(unsigned)ceil_div(n * nrhs, 256), 256, 0, s>>>(B, ldb, X, ldb, perm, n, nrhs);
        B2M_LAUNCHED(ctx);
        if (nrhs <= 64) {  // few right-hand sides: block-row sweeps (dtrsv.cu)
            return tri_solve2_f64(ctx, s, LU, ld, n, kTriL, kTriU, B, ldb, nrhs);
        }
        TriSolve t{LU, ld, n, B, ldb, n, nrhs, 0, nrhs};
        B2M_TRY(trsm_lower_rec(ctx, s, t, 0, 0, n));
        return trsm_upper_rec(ctx, s, t, 0, 0, n);
    });
}

int32_t perm_from_ipiv(Ctx* ctx, cudaStream_t st, const int32_t* ipiv, int64_t n, int32_t* perm) {
    if (n > (1 << 30)) return fail(ctx, B2M_ERR_UNSUPPORTED, "perm_from_ipiv: n too large");
    const size_t smem = (size_t)n * sizeof(int32_t);
    const bool in_smem = smem <= ctx->smem_optin;
    if (in_smem && smem > 48 * 1024) {
        std::atomic<int>& set = device_flag((const void*)perm_from_ipiv_kernel, 0, ctx->device);
        if (!set.load()) {
            B2M_CU(ctx, cudaFuncSetAttribute(perm_from_ipiv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)ctx->smem_optin));
            set.store(1);
        }
    }
    perm_from_ipiv_kernel<<<1, 1024, in_smem ? smem : 0, st>>>(ipiv, (int)n, perm, in_smem ? 1 : 0);
    B2M_LAUNCHED(ctx);
    return B2M_OK;
}

int32_t lu_determinant(Ctx* ctx, cudaStream_t st, const double* LU, int64_t ld, int64_t n, const int32_t* ipiv,
                       double* d_det) {
    if (n > (1 << 30)) return fail(ctx, B2M_ERR_UNSUPPORTED, "determinant: n too large");
    determinant_kernel<<<1, kDetChunk, 0, st>>>(LU, ld, (int)n, ipiv, ctx->d_status, d_det);
    B2M_LAUNCHED(ctx);
    return B2M_OK;
}

int32_t copy_matrix(Ctx* ctx, cudaStream_t st, double* dst, int64_t ldd_bytes, const double* src, int64_t lds_bytes,
                    int64_t rows, int64_t cols) {
    if (rows <= 0 || cols <= 0) return B2M_OK;
    B2M_CU(ctx, cudaMemcpy2DAsync(dst, ldd_bytes, src, lds_bytes, cols * 8, rows, cudaMemcpyDeviceToDevice, st));
    return B2M_OK;
}

}  // namespace b2m

namespace b2m {

__global__ void axpy_matrix_kernel(double* X, int64_t ldx, const double* R, int64_t ldr, int64_t rows, int64_t cols,
                                   const int32_t* status) {
    if (status[kInfo] != 0) return;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= rows * cols) return;
    const int64_t i = e / cols, c = e - i * cols;
    X[i * ldx + c] += R[i * ldr + c];
}

__global__ void set_diagonal_kernel(double* X, int64_t ldx, int64_t n, double v) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) X[i * ldx + i] = v;
}

__global__ void copy_if_ok_kernel(double* dst, int64_t ldd, const double* src, int64_t lds, int64_t rows, int64_t cols,
                                  const int32_t* status) {
    if (status[kInfo] != 0) return;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= rows * cols) return;
    const int64_t i = e / cols, c = e - i * cols;
    dst[i * ldd + c] = src[i * lds + c];
}

__global__ void publish_status_kernel(const int32_t* words, int32_t* out) {
    *out = words[kTimeout] != 0 ? B2M_ERR_TIMEOUT : words[kInfo];
}

int32_t publish_status(Ctx* ctx, cudaStream_t st, const int32_t* words, int32_t* out) {
    publish_status_kernel<<<1, 1, 0, st>>>(words, out);
    B2M_LAUNCHED(ctx);
    return B2M_OK;
}

int32_t axpy_matrix(Ctx* ctx, cudaStream_t st, double* X, int64_t ldx, const double* R, int64_t ldr, int64_t rows,
                    int64_t cols) {
    if (rows <= 0 || cols <= 0) return B2M_OK;
    axpy_matrix_kernel<<<(unsigned)ceil_div(rows * cols, 256), 256, 0, st>>>(X, ldx, R, ldr, rows, cols,
                                                                             ctx->d_status);
    B2M_LAUNCHED(ctx);
    return B2M_OK;
}

int32_t set_diagonal(Ctx* ctx, cudaStream_t st, double* X, int64_t ldx, int64_t n, double v) {
    if (n <= 0) return B2M_OK;
    set_diagonal_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, st>>>(X, ldx, n, v);
    B2M_LAUNCHED(ctx);
    return B2M_OK;
}

int32_t copy_if_ok(Ctx* ctx, cudaStream_t st, double* dst, int64_t ldd, const double* src, int64_t lds, int64_t rows,
                   int64_t cols) {
    if (rows <= 0 || cols <= 0) return B2M_OK;
    copy_if_ok_kernel<<<(unsigned)ceil_div(rows * cols, 256), 256, 0, st>>>(dst, ldd, src, lds, rows, cols,
                                                                           ctx->d_status);
    B2M_LAUNCHED(ctx);
    return B2M_OK;
}

}  // namespace b2m
