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

}  // namespace

int32_t tri_solve_f64(Ctx* ctx, cudaStream_t st, const double* LU, int64_t ld, int64_t n, int mode, double* X,
                      int64_t ldx, int64_t nrhs) {
    if (n <= 0 || nrhs <= 0) return B2M_OK;
    switch (mode) {
        case kTriL: return launch_sweeps<kTriL>(ctx, st, LU, ld, n, X, ldx, nrhs);
        case kTriU: return launch_sweeps<kTriU>(ctx, st, LU, ld, n, X, ldx, nrhs);
        case kTriUt: return launch_sweeps<kTriUt>(ctx, st, LU, ld, n, X, ldx, nrhs);
        case kTriLt: return launch_sweeps<kTriLt>(ctx, st, LU, ld, n, X, ldx, nrhs);
    }
    return fail(ctx, B2M_ERR_ARG, "tri_solve_f64: unknown triangle %d", mode);
}

}  // namespace b2m
