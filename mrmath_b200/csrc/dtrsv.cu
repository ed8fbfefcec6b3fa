// dtrsv.cu -- blocked FP64 triangular solves with a few right-hand sides, on the factors of the
// FP64 LU (unit-lower L below the diagonal, U on and above it, one row-major array).
//
// Four triangles are served by one kernel: L (forward, unit), U (backward, true division by the
// diagonal as in the reference's back substitution, LinAlgLU.pas:362-382), and the transposes
// U^T (forward, division) and L^T (backward, unit) that the adjoint solve A^T lambda = g needs.
//
// One launch per 128-row block b, in sweep order.  The block's diagonal CTAs (four right-hand
// sides each) subtract the previous block's contribution, then solve the 128 x 128 diagonal
// triangle by substitution in four 32-row steps: one warp per right-hand side holds 32 unknowns
// (lane = row), broadcasts each finished unknown with a shuffle, and all warps then fold the 32
// finished unknowns into the rows still to come.  The other CTAs subtract the previous block's
// contribution from every row outside blocks <= b (forward) or >= b (backward), 64 rows each.
// The transposed triangles read the factors column-wise, which is coalesced across the rows a
// warp handles.
#include <algorithm>

#include "common.cuh"
#include "kernels.cuh"

namespace b2m {
namespace {

constexpr int kDtNB = 128;     // rows per block
constexpr int kDtRhs = 4;      // right-hand sides per diagonal CTA
constexpr int kDtRows = 64;    // rows per update CTA
constexpr int kDtMaxRhs = 16;  // right-hand sides per launch

struct DtArgs {
    const double* LU;
    int64_t ld;
    int n;
    double* X;  // n x nrhs, row stride ldx; columns [c0, c0 + nc)
    int64_t ldx;
    int c0, nc;
    int nd;  // diagonal CTAs
    const int32_t* status;
};

// element (i, j) of the triangle being solved
template <int MODE>
__device__ __forceinline__ double tri_at(const double* LU, int64_t ld, int i, int j) {
    return (MODE == kTriL || MODE == kTriU) ? __ldg(LU + (int64_t)i * ld + j) : __ldg(LU + (int64_t)j * ld + i);
}
template <int MODE> __host__ __device__ constexpr bool tri_lower() { return MODE == kTriL || MODE == kTriUt; }
template <int MODE> __host__ __device__ constexpr bool tri_unit() { return MODE == kTriL || MODE == kTriLt; }

template <int MODE>
__global__ void __launch_bounds__(256) dtrsv_block_kernel(DtArgs a, int b) {
    __shared__ double s_p[kDtNB][kDtMaxRhs + 1];  // solution of the previous block
    __shared__ double s_y[kDtNB][kDtRhs + 1];
    __shared__ double s_h[kDtNB][kDtRhs + 1];
    if (a.status[kInfo] != 0) return;
    constexpr bool lower = tri_lower<MODE>();
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int nblk = (int)ceil_div(a.n, kDtNB);
    const int prev = lower ? b - 1 : b + 1;
    const bool has_prev = prev >= 0 && prev < nblk;
    const int p0 = prev * kDtNB, ps = has_prev ? min(kDtNB, a.n - p0) : 0;
    const int b0 = b * kDtNB, bs = min(kDtNB, a.n - b0);
    if (blockIdx.x < a.nd) {
        const int g = blockIdx.x * kDtRhs;
        // y = X_b - T(b, prev) X_prev: thread (row r, half h) sums 64 of the 128 previous unknowns
        for (int e = t; e < kDtNB * kDtRhs; e += 256) {
            const int k = e >> 2, q = e & 3;
            s_p[k][q] = (k < ps && g + q < a.nc) ? a.X[(int64_t)(p0 + k) * a.ldx + a.c0 + g + q] : 0.0;
        }
        __syncthreads();
        const int r = t & (kDtNB - 1), h = t >> 7;
        double acc[kDtRhs] = {0.0, 0.0, 0.0, 0.0};
        if (r < bs) {
            // all 64 loads of this thread's half row are in flight before the first product (same
            // ascending order of contributions as one load per step)
#pragma unroll
            for (int k2 = 0; k2 < 64; k2 += 32) {
                double tv[32];
#pragma unroll
                for (int kk = 0; kk < 32; ++kk) {
                    const int k = 64 * h + k2 + kk;
                    tv[kk] = k < ps ? tri_at<MODE>(a.LU, a.ld, b0 + r, p0 + k) : 0.0;
                }
#pragma unroll
                for (int kk = 0; kk < 32; ++kk) {
                    const int k = 64 * h + k2 + kk;
                    if (k < ps) {
#pragma unroll
                        for (int q = 0; q < kDtRhs; ++q) acc[q] = fma(tv[kk], s_p[k][q], acc[q]);
                    }
                }
            }
        }
        if (h == 1) {
#pragma unroll
            for (int q = 0; q < kDtRhs; ++q) s_h[r][q] = acc[q];
        }
        __syncthreads();
        if (h == 0) {
#pragma unroll
            for (int q = 0; q < kDtRhs; ++q) {
                const bool ok = r < bs && g + q < a.nc;
                s_y[r][q] = ok ? a.X[(int64_t)(b0 + r) * a.ldx + a.c0 + g + q] - (acc[q] + s_h[r][q]) : 0.0;
            }
        }
        __syncthreads();
        // substitution on the diagonal triangle, 32 rows at a time
        const int nsub = (bs + 31) / 32;
        for (int si = 0; si < nsub; ++si) {
            const int s = lower ? si : nsub - 1 - si;
            const int s0 = 32 * s, sw = min(32, bs - s0);
            if (warp < kDtRhs) {
                const int q = warp;
                double tr[32];
#pragma unroll
                for (int j = 0; j < 32; ++j)
                    tr[j] = (lane < sw && j < sw) ? tri_at<MODE>(a.LU, a.ld, b0 + s0 + lane, b0 + s0 + j) : 0.0;
                double y = lane < sw ? s_y[s0 + lane][q] : 0.0;
                if (lower) {
#pragma unroll
                    for (int j = 0; j < 32; ++j) {
                        if (j >= sw) break;
                        if (!tri_unit<MODE>() && lane == j) y = y / tr[j];
                        const double xj = __shfl_sync(0xffffffffu, y, j);
                        if (lane > j) y = fma(-tr[j], xj, y);
                    }
                } else {
#pragma unroll
                    for (int j = 31; j >= 0; --j) {
                        if (j >= sw) continue;
                        if (!tri_unit<MODE>() && lane == j) y = y / tr[j];
                        const double xj = __shfl_sync(0xffffffffu, y, j);
                        if (lane < j) y = fma(-tr[j], xj, y);
                    }
                }
                if (lane < sw) s_y[s0 + lane][q] = y;
            }
            __syncthreads();
            // fold the 32 finished unknowns into the rows of this block still to be solved
            const int rlo = lower ? s0 + sw : 0, rhi = lower ? bs : s0;
            for (int e = t; e < (rhi - rlo) * kDtRhs; e += 256) {
                const int rr = rlo + (e >> 2), q = e & 3;
                double tv[32];
#pragma unroll
                for (int j = 0; j < 32; ++j) tv[j] = j < sw ? tri_at<MODE>(a.LU, a.ld, b0 + rr, b0 + s0 + j) : 0.0;
                double acc2 = 0.0;
#pragma unroll
                for (int j = 0; j < 32; ++j)
                    if (j < sw) acc2 = fma(tv[j], s_y[s0 + j][q], acc2);
                s_y[rr][q] -= acc2;
            }
            __syncthreads();
        }
        for (int e = t; e < bs * kDtRhs; e += 256) {
            const int rr = e >> 2, q = e & 3;
            if (g + q < a.nc) a.X[(int64_t)(b0 + rr) * a.ldx + a.c0 + g + q] = s_y[rr][q];
        }
        return;
    }
    if (!has_prev) return;
    // update CTA: rows [u0, u0 + 64) of the rows still to come; 4 lanes per row split K in quarters
    const int u = blockIdx.x - a.nd;
    const int u0 = lower ? b0 + bs + u * kDtRows : u * kDtRows;
    const int uend = lower ? a.n : b0;
    if (u0 >= uend) return;
    for (int e = t; e < ps * a.nc; e += 256) {
        const int k = e / a.nc, c = e - k * a.nc;
        s_p[k][c] = a.X[(int64_t)(p0 + k) * a.ldx + a.c0 + c];
    }
    __syncthreads();
    const int rr = t >> 2, kq = t & 3;
    const int row = u0 + rr;
    double acc[kDtMaxRhs];
#pragma unroll
    for (int c = 0; c < kDtMaxRhs; ++c) acc[c] = 0.0;
    if (row < uend) {
        double tv[32];  // all loads in flight before the first product
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            const int k = 4 * i + kq;  // interleaved quarters: the four lanes of a row read adjacent k
            tv[i] = k < ps ? tri_at<MODE>(a.LU, a.ld, row, p0 + k) : 0.0;
        }
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            const int k = 4 * i + kq;
            if (k < ps) {
#pragma unroll
                for (int c = 0; c < kDtMaxRhs; ++c)
                    if (c < a.nc) acc[c] = fma(tv[i], s_p[k][c], acc[c]);
            }
        }
    }
#pragma unroll
    for (int c = 0; c < kDtMaxRhs; ++c) {
        acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], 1);
        acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], 2);
    }
    if (row < uend) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int c = 4 * kq + i;  // lane kq of the row writes columns 4 kq .. 4 kq + 3
            const double v = kq == 0 ? acc[i] : kq == 1 ? acc[4 + i] : kq == 2 ? acc[8 + i] : acc[12 + i];
            if (c < a.nc) a.X[(int64_t)row * a.ldx + a.c0 + c] -= v;
        }
    }
}

template <int MODE>
int32_t launch_sweeps(Ctx* ctx, cudaStream_t st, const double* LU, int64_t ld, int64_t n, double* X, int64_t ldx,
                      int64_t nrhs) {
    constexpr bool lower = tri_lower<MODE>();
    const int nblk = (int)ceil_div(n, kDtNB);
    for (int64_t c0 = 0; c0 < nrhs; c0 += kDtMaxRhs) {
        const int nc = (int)std::min<int64_t>(kDtMaxRhs, nrhs - c0);
        DtArgs a{LU, ld, (int)n, X, ldx, (int)c0, nc, (int)ceil_div(nc, kDtRhs), ctx->d_status};
        for (int i = 0; i < nblk; ++i) {
            const int b = lower ? i : nblk - 1 - i;
            const int64_t rows = lower ? n - std::min<int64_t>(n, (int64_t)(b + 1) * kDtNB) : (int64_t)b * kDtNB;
            const int nu = i > 0 ? (int)ceil_div(rows, kDtRows) : 0;
            prof_begin(ctx, st, kClsSolve);
            dtrsv_block_kernel<MODE><<<a.nd + nu, 256, 0, st>>>(a, b);
            prof_end(ctx, st, kClsSolve, 8.0 * kDtNB * (rows + kDtNB) + 16.0 * (rows + kDtNB) * nc);
            B2M_LAUNCHED(ctx);
        }
    }
    return B2M_OK;
}

// ---- One persistent launch per sweep (orders > 128).  The triangle is cut into 64-row blocks;
// each diagonal block's inverse (substitution by columns of the identity, with the true division
// for U and U^T) and each coupling block W_b = T_bb^-1 T_{b,p} (p the block before b in sweep
// order) are formed first, then a CTA per (block, 8 right-hand sides) folds in the earlier blocks
// as they are published and finishes x_b = T_bb^-1 y_b - W_b x_p, so one 64 x 64 x 8 product per
// block is on the chain.  A block is published as 512 doubles over words preset to an empty
// pattern (all bits set, which no arithmetic result has): each 64-bit store carries its own
// readiness, so there is neither a fence nor a flag round trip; every wait is bounded and a CTA
// that gives up writes the abort pattern so that its dependants stop at once.
constexpr int kDsNB = 64;
constexpr int kDsRhs = 8;
constexpr int kDsThreads = 128;
constexpr int kDsMaxRhs = 16;  // right-hand sides per sweep launch
constexpr int kDsTS = kDsNB + 2;  // line stride of the staged T_bj (528 bytes: 16-byte aligned lines)
constexpr int kDsSmem = (2 * kDsNB * kDsNB + kDsNB * kDsTS) * (int)sizeof(double);  // T_bb^-1, W_b, T_bj
constexpr int kDsTriSmem = 2 * kDsNB * (kDsNB + 1) * (int)sizeof(double);
constexpr uint32_t kDsSpin = 1u << 22;
constexpr unsigned long long kDsEmpty = ~0ull;        // a word not yet published
constexpr unsigned long long kDsAbort = ~0ull - 1ull;  // a block whose CTA gave up

__device__ __forceinline__ unsigned long long ds_ld64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];\n" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void ds_st64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;\n" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src, int src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}

// T_bj (64 x 64) into shared memory as 64 lines of kDsTS doubles: line r holds row r of T_bj for the
// row-major triangles (L, U), line c holds column c for the transposed ones (U^T, L^T) -- in both
// cases a 512-byte run of one row of the factors.  A full block whose lines are 16-byte aligned
// comes in as 64 bulk copies (one instruction per line) completing on `bar`; otherwise
// asynchronous 8-byte copies, zero past the matrix.  The fold reads column k of T_bj across 32
// consecutive rows with at most four shared-memory wavefronts.
template <int MODE>
__device__ __forceinline__ bool ds_stage(double* s_tt, const double* LU, int64_t ld, int b0, int bs, int p0, int ps,
                                         int t, bool bulk_ok, uint64_t* bar) {
    constexpr bool trans = !(MODE == kTriL || MODE == kTriU);
    if (bulk_ok && bs == kDsNB && ps == kDsNB) {
        if (t == 0) mbar_arrive_expect_tx(bar, kDsNB * kDsNB * (int)sizeof(double));
        if (t < kDsNB) {
            const double* src = trans ? LU + (int64_t)(p0 + t) * ld + b0 : LU + (int64_t)(b0 + t) * ld + p0;
            bulk_g2s(s_tt + t * kDsTS, src, kDsNB * (int)sizeof(double), bar);
        }
        return true;
    }
#pragma unroll 8
    for (int i = 0; i < kDsNB * kDsNB / kDsThreads; ++i) {
        const int e = t + kDsThreads * i;
        const int line = e / kDsNB, pos = e & (kDsNB - 1);  // pos runs along the factors' row
        const int rr = trans ? pos : line, cc = trans ? line : pos;
        const bool in = rr < bs && cc < ps;
        const double* src = trans ? LU + (int64_t)(p0 + cc) * ld + b0 + rr : LU + (int64_t)(b0 + rr) * ld + p0 + cc;
        cp_async8(s_tt + line * kDsTS + pos, in ? src : LU, in ? 8 : 0);
    }
    cp_async_commit();
    return false;
}

// inverse of the diagonal block b of the triangle (thread per column; zero past the matrix)
template <int MODE>
__global__ void __launch_bounds__(kDsNB) dinv_kernel(const double* LU, int64_t ld, int n, double* inv,
                                                     const int32_t* status) {
    extern __shared__ double dt_sm[];
    if (status[kInfo] != 0) return;
    constexpr bool lower = tri_lower<MODE>(), unit = tri_unit<MODE>();
    const int b = blockIdx.x, b0 = b * kDsNB, bs = min(kDsNB, n - b0), c = threadIdx.x;
    constexpr int SP = kDsNB + 1;
    double* s_t = dt_sm;
    double* s_x = dt_sm + kDsNB * SP;
    batched_copy<1, 16, double>(0, kDsNB,
        [&](int r) { return (r < bs && c < bs) ? tri_at<MODE>(LU, ld, b0 + r, b0 + c) : 0.0; },
        [&](int r, double v) { s_t[r * SP + c] = v; });
    __syncthreads();
    if (lower) {
        for (int i = 0; i < kDsNB; ++i) {
            double acc = (i == c) ? 1.0 : 0.0;
            if (i < bs && c < bs) {
                for (int k = c; k < i; ++k) acc = fma(-s_t[i * SP + k], s_x[k * SP + c], acc);
                if (!unit && i >= c) acc = acc / s_t[i * SP + i];
            }
            s_x[i * SP + c] = (i < bs && c < bs && i >= c) ? acc : 0.0;
        }
    } else {
        for (int i = kDsNB - 1; i >= 0; --i) {
            double acc = (i == c) ? 1.0 : 0.0;
            if (i < bs && c < bs) {
                for (int k = i + 1; k <= c; ++k) acc = fma(-s_t[i * SP + k], s_x[k * SP + c], acc);
                if (!unit && i <= c) acc = acc / s_t[i * SP + i];
            }
            s_x[i * SP + c] = (i < bs && c < bs && i <= c) ? acc : 0.0;
        }
    }
    __syncthreads();
    double* out = inv + (int64_t)b * kDsNB * kDsNB;
    for (int r = 0; r < kDsNB; ++r) out[r * kDsNB + c] = s_x[r * SP + c];
}

// W_b = T_bb^-1 T_{b,p} for every block b with a predecessor p in sweep order (zero past the matrix)
template <int MODE>
__global__ void __launch_bounds__(256) dcouple_kernel(const double* LU, int64_t ld, int n, const double* inv, double* w,
                                                      const int32_t* status) {
    extern __shared__ double dc_sm[];
    if (status[kInfo] != 0) return;
    constexpr bool lower = tri_lower<MODE>();
    const int nblk = (int)ceil_div(n, kDsNB);
    const int b = blockIdx.x;
    if (lower ? b == 0 : b == nblk - 1) return;
    const int b0 = b * kDsNB, bs = min(kDsNB, n - b0);
    const int p0 = lower ? b0 - kDsNB : b0 + kDsNB, ps = min(kDsNB, n - p0);
    constexpr int SP = kDsNB + 1;
    double* s_i = dc_sm;
    double* s_t = dc_sm + kDsNB * SP;
    const int t = threadIdx.x;
    batched_copy<256, 8, double>(t, kDsNB * kDsNB, [&](int e) { return inv[(int64_t)b * kDsNB * kDsNB + e]; },
                                 [&](int e, double v) { s_i[(e / kDsNB) * SP + e % kDsNB] = v; });
    batched_copy<256, 8, double>(t, kDsNB * kDsNB,
        [&](int e) {
            const int r = e / kDsNB, c = e % kDsNB;
            return (r < bs && c < ps) ? tri_at<MODE>(LU, ld, b0 + r, p0 + c) : 0.0;
        },
        [&](int e, double v) { s_t[(e / kDsNB) * SP + e % kDsNB] = v; });
    __syncthreads();
    const int r0 = 4 * (t >> 4), c0 = t & 15;
    double acc[4][4] = {};
    for (int k = 0; k < kDsNB; ++k) {
        double iv[4], tv[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) iv[i] = s_i[(r0 + i) * SP + k];
#pragma unroll
        for (int j = 0; j < 4; ++j) tv[j] = s_t[k * SP + c0 + 16 * j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = fma(iv[i], tv[j], acc[i][j]);
    }
    double* out = w + (int64_t)b * kDsNB * kDsNB;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) out[(r0 + i) * kDsNB + c0 + 16 * j] = acc[i][j];
}

struct DsArgs {
    const double* LU;
    int64_t ld;
    int n;
    const double* inv;  // [nblk][64][64]
    const double* w;    // [nblk][64][64]
    double* X;
    int64_t ldx;
    int c0, nc;
    unsigned long long* pub;  // [nblk][ng][64][8] published blocks (double bits; preset to kDsEmpty)
    int32_t* status;
    uint32_t spin;
    bool bulk;  // the factors' rows are 16-byte aligned: full blocks are staged by bulk copies
};

template <int MODE>
__global__ void __launch_bounds__(kDsThreads) dsweep_kernel(DsArgs a) {
    extern __shared__ __align__(16) double ds_dyn[];
    __shared__ double s_p[kDsNB][kDsRhs + 1];  // x of the block being folded in
    __shared__ double s_y[kDsNB][kDsRhs + 1];
    __shared__ double s_h[kDsNB][kDsRhs + 1];  // second-half partial sums
    __shared__ int s_abort;
    double* s_inv = ds_dyn;                    // [k][r]: T_bb^-1 transposed
    double* s_w = ds_dyn + kDsNB * kDsNB;      // [k][r]: W_b transposed
    double* s_tt = ds_dyn + 2 * kDsNB * kDsNB; // T_bj of the block being folded in (kDsNB lines of kDsTS)
    __shared__ __align__(8) uint64_t s_tbar;   // completion of a bulk-staged T_bj
    if (a.status[kInfo] != 0) return;
    constexpr bool lower = tri_lower<MODE>();
    const int t = threadIdx.x, r = t & (kDsNB - 1), h = t >> 6;
    const int nblk = (int)ceil_div(a.n, kDsNB), ng = (int)ceil_div(a.nc, kDsRhs);
    const int bi = blockIdx.x / ng, g = blockIdx.x - bi * ng;
    const int b = lower ? bi : nblk - 1 - bi;
    const int b0 = b * kDsNB, bs = min(kDsNB, a.n - b0);
    const int cg = a.c0 + g * kDsRhs, ncg = min(kDsRhs, a.nc - g * kDsRhs);
    for (int e = t; e < kDsNB * kDsNB; e += kDsThreads) {  // row-major blocks, stored transposed
        const int rr = e / kDsNB, k = e - rr * kDsNB;
        s_inv[k * kDsNB + rr] = a.inv[(int64_t)b * kDsNB * kDsNB + e];
        if (bi > 0) s_w[k * kDsNB + rr] = a.w[(int64_t)b * kDsNB * kDsNB + e];
    }
    double xb[kDsRhs], acc[kDsRhs];
#pragma unroll
    for (int q = 0; q < kDsRhs; ++q) {
        xb[q] = (h == 0 && r < bs && q < ncg) ? a.X[(int64_t)(b0 + r) * a.ldx + cg + q] : 0.0;
        acc[q] = 0.0;
    }
    if (t == 0) {
        s_abort = 0;
        mbar_init(&s_tbar, 1);
        fence_barrier_init();
    }
    __syncthreads();
    uint32_t tphase = 0;
    constexpr bool trans = !(MODE == kTriL || MODE == kTriU);
    // block j published: its 64 x 8 values into s_p (thread t polls words t, t + 128, ...); also
    // completes this thread's part of a staged T_bj (the bulk copies even when the wait gives up, so
    // that no copy is in flight when the CTA leaves)
    auto wait_block = [&](int j, bool bulk_staged) -> bool {
        const unsigned long long* src = a.pub + (size_t)(j * ng + g) * (kDsNB * kDsRhs);
        unsigned long long w[4];
        bool ready = false, bad = false;
        for (uint32_t it = 0; it < a.spin && !ready && !bad; ++it) {
            ready = true;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                w[e] = ds_ld64(src + t + kDsThreads * e);
                ready = ready && w[e] != kDsEmpty;
                bad = bad || w[e] == kDsAbort;
            }
            if (!ready && (it & 255u) == 255u && *reinterpret_cast<volatile int32_t*>(&a.status[kTimeout]) != 0)
                bad = true;
        }
        if (!ready && !bad) atomicCAS(&a.status[kTimeout], 0, 505);
        if (!ready || bad) s_abort = 1;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int idx = t + kDsThreads * e;
            s_p[idx >> 3][idx & 7] = __longlong_as_double((long long)w[e]);
        }
        cp_async_wait<0>();  // this thread's part of T_bj has landed
        if (bulk_staged) {
            if (!mbar_wait(&s_tbar, tphase, &a.status[kTimeout], 506)) s_abort = 1;
            tphase ^= 1u;
        }
        __syncthreads();
        return !s_abort;
    };
    bool ok = true;
    for (int jj = 0; ok && jj + 1 < bi; ++jj) {
        const int j = lower ? jj : nblk - 1 - jj;
        const int p0 = j * kDsNB, ps = min(kDsNB, a.n - p0);
        // T_bj is staged while this CTA waits for x_j
        const bool bulk = ds_stage<MODE>(s_tt, a.LU, a.ld, b0, bs, p0, ps, t, a.bulk, &s_tbar);
        ok = wait_block(j, bulk);
        if (!ok) break;
#pragma unroll
        for (int k = 0; k < 32; ++k) {
            const int kk = 32 * h + k;
            const double tv = trans ? s_tt[kk * kDsTS + r] : s_tt[r * kDsTS + kk];
#pragma unroll
            for (int q = 0; q < kDsRhs; ++q) acc[q] = fma(tv, s_p[32 * h + k][q], acc[q]);
        }
        __syncthreads();  // s_p is rewritten by the next wait
    }
    if (ok) {
        // y = X_b - sum T_bj x_j ;  z = T_bb^-1 y
        if (h == 1) {
#pragma unroll
            for (int q = 0; q < kDsRhs; ++q) s_h[r][q] = acc[q];
        }
        __syncthreads();
        if (h == 0) {
#pragma unroll
            for (int q = 0; q < kDsRhs; ++q) s_y[r][q] = xb[q] - acc[q] - s_h[r][q];
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < kDsRhs; ++q) acc[q] = 0.0;
#pragma unroll 8
        for (int k = 0; k < 32; ++k) {
            const int kk = 32 * h + k;
            const double m = s_inv[kk * kDsNB + r];
#pragma unroll
            for (int q = 0; q < kDsRhs; ++q) acc[q] = fma(m, s_y[kk][q], acc[q]);
        }
        if (bi > 0) {  // x_b = z - W_b x_p
            ok = wait_block(lower ? b - 1 : b + 1, false);
            if (ok) {
#pragma unroll 8
                for (int k = 0; k < 32; ++k) {
                    const int kk = 32 * h + k;
                    const double m = s_w[kk * kDsNB + r];
#pragma unroll
                    for (int q = 0; q < kDsRhs; ++q) acc[q] = fma(-m, s_p[kk][q], acc[q]);
                }
            }
        }
    }
    if (ok) {
        if (h == 1) {
#pragma unroll
            for (int q = 0; q < kDsRhs; ++q) s_h[r][q] = acc[q];
        }
        __syncthreads();
        if (h == 0) {
            unsigned long long* dst = a.pub + (size_t)(b * ng + g) * (kDsNB * kDsRhs) + r * kDsRhs;
#pragma unroll
            for (int q = 0; q < kDsRhs; ++q) {
                const double xv = (r < bs && q < ncg) ? acc[q] + s_h[r][q] : 0.0;
                unsigned long long bits = (unsigned long long)__double_as_longlong(xv);
                if (bits >= kDsAbort) bits = 0x7FF8000000000000ull;  // a NaN carrying a reserved pattern
                ds_st64(dst + q, bits);
                if (r < bs && q < ncg) a.X[(int64_t)(b0 + r) * a.ldx + cg + q] = xv;
            }
        }
    } else {  // dependants stop at once
        unsigned long long* dst = a.pub + (size_t)(b * ng + g) * (kDsNB * kDsRhs);
#pragma unroll
        for (int e = 0; e < 4; ++e) ds_st64(dst + t + kDsThreads * e, kDsAbort);
    }
}

// whether the persistent sweep of this triangle can run for nrhs right-hand sides (every CTA
// co-resident with the others); sets the kernels' shared-memory attributes once per device
template <int MODE>
int32_t chain_usable(Ctx* ctx, int64_t n, int64_t nrhs, bool* usable) {
    *usable = false;
    if (n <= 2 * kDsNB) return B2M_OK;
    std::atomic<int>& attr = device_flag((const void*)dsweep_kernel<MODE>, 0, ctx->device);
    if (!attr.load()) {
        B2M_CU(ctx, cudaFuncSetAttribute(dsweep_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, kDsSmem));
        B2M_CU(ctx, cudaFuncSetAttribute(dinv_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, kDsTriSmem));
        B2M_CU(ctx, cudaFuncSetAttribute(dcouple_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, kDsTriSmem));
        attr.store(1);
    }
    if (ctx->dsweep_ctas < 0) {
        int per_sm = 0, coop = 0;
        B2M_CU(ctx, cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, ctx->device));
        B2M_CU(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dsweep_kernel<MODE>, kDsThreads, kDsSmem));
        ctx->dsweep_ctas = coop ? per_sm * ctx->num_sms : 0;
    }
    const int nblk = (int)ceil_div(n, kDsNB);
    const int ngmax = (int)ceil_div(std::min<int64_t>(nrhs, kDsMaxRhs), kDsRhs);
    *usable = (int64_t)nblk * ngmax <= ctx->dsweep_ctas;
    return B2M_OK;
}

size_t chain_blk_doubles(int64_t n) { return (size_t)ceil_div(n, kDsNB) * kDsNB * kDsNB; }
size_t chain_pub_doubles(int64_t n) { return (size_t)ceil_div(n, kDsNB) * 2 * kDsNB * kDsRhs; }

// the diagonal-block inverses and coupling blocks of the sweep
template <int MODE>
int32_t chain_prepare(Ctx* ctx, cudaStream_t st, const double* LU, int64_t ld, int64_t n, double* inv, double* w) {
    const int nblk = (int)ceil_div(n, kDsNB);
    const size_t blk_doubles = chain_blk_doubles(n);
    prof_begin(ctx, st, kClsSolve);
    dinv_kernel<MODE><<<nblk, kDsNB, kDsTriSmem, st>>>(LU, ld, (int)n, inv, ctx->d_status);
    prof_end(ctx, st, kClsSolve, 8.0 * 2 * blk_doubles);
    B2M_LAUNCHED(ctx);
    prof_begin(ctx, st, kClsSolve);
    dcouple_kernel<MODE><<<nblk, 256, kDsTriSmem, st>>>(LU, ld, (int)n, inv, w, ctx->d_status);
    prof_end(ctx, st, kClsSolve, 8.0 * 3 * blk_doubles);
    B2M_LAUNCHED(ctx);
    return B2M_OK;
}

// the persistent sweeps (one cooperative launch per kDsMaxRhs right-hand sides)
template <int MODE>
int32_t chain_sweeps(Ctx* ctx, cudaStream_t st, const double* LU, int64_t ld, int64_t n, const double* inv,
                     const double* w, unsigned long long* pub, double* X, int64_t ldx, int64_t nrhs) {
    const int nblk = (int)ceil_div(n, kDsNB);
    for (int64_t c0 = 0; c0 < nrhs; c0 += kDsMaxRhs) {
        const int nc = (int)std::min<int64_t>(kDsMaxRhs, nrhs - c0);
        const int ng = (int)ceil_div(nc, kDsRhs);
        B2M_CU(ctx, cudaMemsetAsync(pub, 0xFF, (size_t)nblk * ng * kDsNB * kDsRhs * sizeof(double), st));  // kDsEmpty
        DsArgs da{LU, ld, (int)n, inv, w, X, ldx, (int)c0, nc, pub, ctx->d_status,
                  ctx->wait_limit >= 0 ? (uint32_t)ctx->wait_limit : kDsSpin, aligned16(LU) && ld % 2 == 0};
        cudaLaunchConfig_t cfg{};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeCooperative;
        at[0].val.cooperative = 1;
        cfg.gridDim = dim3((unsigned)(nblk * ng));
        cfg.blockDim = dim3(kDsThreads);
        cfg.dynamicSmemBytes = kDsSmem;
        cfg.stream = st;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        prof_begin(ctx, st, kClsSolve);
        B2M_CU(ctx, cudaLaunchKernelEx(&cfg, dsweep_kernel<MODE>, da));
        prof_end(ctx, st, kClsSolve, 4.0 * (double)n * n + 16.0 * n * nc);
        B2M_LAUNCHED(ctx);
    }
    return B2M_OK;
}

template <int MODE>
int32_t launch_chain(Ctx* ctx, cudaStream_t st, const double* LU, int64_t ld, int64_t n, double* X, int64_t ldx,
                     int64_t nrhs, bool* used) {
    B2M_TRY(chain_usable<MODE>(ctx, n, nrhs, used));
    if (!*used) return B2M_OK;  // not co-resident: per-block launches
    const size_t blk_doubles = chain_blk_doubles(n);
    void* p = nullptr;
    B2M_TRY(ws_get(ctx, kWsTri, (2 * blk_doubles + chain_pub_doubles(n)) * sizeof(double), &p));
    double* inv = static_cast<double*>(p);
    double* w = inv + blk_doubles;
    unsigned long long* pub = reinterpret_cast<unsigned long long*>(w + blk_doubles);
    B2M_TRY(chain_prepare<MODE>(ctx, st, LU, ld, n, inv, w));
    return chain_sweeps<MODE>(ctx, st, LU, ld, n, inv, w, pub, X, ldx, nrhs);
}

// two sweeps in sequence; the second triangle's blocks are prepared on the side stream meanwhile
template <int M1, int M2>
int32_t solve_pair(Ctx* ctx, cudaStream_t st, const double* LU, int64_t ld, int64_t n, double* X, int64_t ldx,
                   int64_t nrhs, bool* used) {
    bool u1 = false, u2 = false;
    B2M_TRY(chain_usable<M1>(ctx, n, nrhs, &u1));
    B2M_TRY(chain_usable<M2>(ctx, n, nrhs, &u2));
    *used = u1 && u2;
    if (!*used) return B2M_OK;
    B2M_TRY(ensure_side_stream(ctx));
    const size_t blk_doubles = chain_blk_doubles(n);
    void* p = nullptr;
    B2M_TRY(ws_get(ctx, kWsTri, (4 * blk_doubles + chain_pub_doubles(n)) * sizeof(double), &p));
    double* inv1 = static_cast<double*>(p);
    double* w1 = inv1 + blk_doubles;
    double* inv2 = w1 + blk_doubles;
    double* w2 = inv2 + blk_doubles;
    unsigned long long* pub = reinterpret_cast<unsigned long long*>(w2 + blk_doubles);
    cudaStream_t q2 = ctx->side_stream;
    B2M_CU(ctx, cudaEventRecord(ctx->ev_side_fork, st));
    B2M_CU(ctx, cudaStreamWaitEvent(q2, ctx->ev_side_fork, 0));
    B2M_TRY(chain_prepare<M2>(ctx, q2, LU, ld, n, inv2, w2));
    B2M_CU(ctx, cudaEventRecord(ctx->ev_side_join, q2));
    B2M_TRY(chain_prepare<M1>(ctx, st, LU, ld, n, inv1, w1));
    // the first sweep is a cooperative launch that needs every SM free of the preparation kernels,
    // so both preparations finish before it starts
    B2M_CU(ctx, cudaStreamWaitEvent(st, ctx->ev_side_join, 0));
    B2M_TRY(chain_sweeps<M1>(ctx, st, LU, ld, n, inv1, w1, pub, X, ldx, nrhs));
    return chain_sweeps<M2>(ctx, st, LU, ld, n, inv2, w2, pub, X, ldx, nrhs);
}

template <int MODE>
int32_t solve_tri(Ctx* ctx, cudaStream_t st, const double* LU, int64_t ld, int64_t n, double* X, int64_t ldx,
                  int64_t nrhs) {
    if (n > 2 * kDsNB) {
        bool used = false;
        B2M_TRY(launch_chain<MODE>(ctx, st, LU, ld, n, X, ldx, nrhs, &used));
        if (used) return B2M_OK;
    }
    return launch_sweeps<MODE>(ctx, st, LU, ld, n, X, ldx, nrhs);
}

}  // namespace

int32_t tri_solve2_f64(Ctx* ctx, cudaStream_t st, const double* LU, int64_t ld, int64_t n, int mode1, int mode2,
                       double* X, int64_t ldx, int64_t nrhs) {
    if (n <= 0 || nrhs <= 0) return B2M_OK;
    bool used = false;
    if (mode1 == kTriL && mode2 == kTriU) B2M_TRY((solve_pair<kTriL, kTriU>(ctx, st, LU, ld, n, X, ldx, nrhs, &used)));
    if (mode1 == kTriUt && mode2 == kTriLt)
        B2M_TRY((solve_pair<kTriUt, kTriLt>(ctx, st, LU, ld, n, X, ldx, nrhs, &used)));
    if (mode1 == kTriUt && mode2 == kTriU) B2M_TRY((solve_pair<kTriUt, kTriU>(ctx, st, LU, ld, n, X, ldx, nrhs, &used)));
    if (used) return B2M_OK;
    B2M_TRY(tri_solve_f64(ctx, st, LU, ld, n, mode1, X, ldx, nrhs));
    return tri_solve_f64(ctx, st, LU, ld, n, mode2, X, ldx, nrhs);
}

int32_t tri_solve_f64(Ctx* ctx, cudaStream_t st, const double* LU, int64_t ld, int64_t n, int mode, double* X,
                      int64_t ldx, int64_t nrhs) {
    if (n <= 0 || nrhs <= 0) return B2M_OK;
    switch (mode) {
        case kTriL: return solve_tri<kTriL>(ctx, st, LU, ld, n, X, ldx, nrhs);
        case kTriU: return solve_tri<kTriU>(ctx, st, LU, ld, n, X, ldx, nrhs);
        case kTriUt: return solve_tri<kTriUt>(ctx, st, LU, ld, n, X, ldx, nrhs);
        case kTriLt: return solve_tri<kTriLt>(ctx, st, LU, ld, n, X, ldx, nrhs);
    }
    return fail(ctx, B2M_ERR_ARG, "tri_solve_f64: unknown triangle %d", mode);
}

}  // namespace b2m
