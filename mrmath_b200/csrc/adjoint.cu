// adjoint.cu -- the adjoint of the LU solve (SolveLinEQAdjoint).  There is no counterpart in the
// reference; it differentiates MatrixLinEQSolve (LinAlgLU.pas:481-592): for X = A^{-1} B and a
// seed G = dL/dX,
//     Lambda = A^{-T} G,   dL/dB = Lambda,   dL/dA = -Lambda X^T.
// With the factors of MatrixLUDecomp (P A = L U, P from the reference's interchange vector indx),
// A^T = U^T L^T P, so Lambda = P^T (L^{-T} (U^{-T} G)): two blocked triangular sweeps over the
// stored factors read column-wise (dtrsv.cu) and a scatter by the permutation.  dA = -Lambda X^T
// is one fused rank-k update: each CTA keeps 16 rows of Lambda in shared memory and streams 256
// columns of dA, so dA is written exactly once (the kernel is bound by that write).
#include "common.cuh"
#include "kernels.cuh"

namespace b2m {
namespace {

constexpr int kRkRows = 16;   // rows of dA per CTA
constexpr int kRkCols = 256;  // columns of dA per CTA (one per thread)
constexpr int kRkK = 32;      // right-hand sides per pass

// Lambda[perm[i]][:] = Y[i][:]
__global__ void scatter_rows_kernel(double* Lam, int64_t ldl, const double* Y, int64_t ldy, const int32_t* perm,
                                    int64_t n, int64_t k, const int32_t* status) {
    if (status[kInfo] != 0) return;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * k) return;
    const int64_t i = e / k, c = e - i * k;
    Lam[(int64_t)perm[i] * ldl + c] = Y[i * ldy + c];
}

// dA[i][j] (op)= -sum_c Lam[i][c] X[j][c] over columns c in [c0, c0 + kc), kc <= KC (the products
// run over KC columns, the ones past kc being zero: KC is the smallest of 1, 4, 32 that holds kc,
// so that a single right-hand side costs one FMA per entry and the kernel stays bound by the write)
template <int KC>
__global__ void __launch_bounds__(kRkCols) rank_update_kernel(double* dA, int64_t ldd, const double* Lam, int64_t ldl,
                                                              const double* X, int64_t ldx, int64_t n, int c0, int kc,
                                                              int accumulate) {
    __shared__ double s_l[kRkRows][KC];
    const int t = threadIdx.x;
    const int64_t i0 = (int64_t)blockIdx.y * kRkRows;
    const int64_t j = (int64_t)blockIdx.x * kRkCols + t;
    for (int e = t; e < kRkRows * KC; e += kRkCols) {
        const int r = e / KC, c = e - r * KC;
        s_l[r][c] = (i0 + r < n && c < kc) ? Lam[(i0 + r) * ldl + c0 + c] : 0.0;
    }
    double xj[KC];
#pragma unroll
    for (int c = 0; c < KC; ++c) xj[c] = (j < n && c < kc) ? X[j * ldx + c0 + c] : 0.0;
    __syncthreads();
    if (j >= n) return;
    double old[kRkRows];
    if (accumulate) {
#pragma unroll
        for (int r = 0; r < kRkRows; ++r) old[r] = i0 + r < n ? dA[(i0 + r) * ldd + j] : 0.0;
    }
#pragma unroll
    for (int r = 0; r < kRkRows; ++r) {
        if (i0 + r >= n) break;
        double acc = 0.0;
#pragma unroll
        for (int c = 0; c < KC; ++c) acc = fma(s_l[r][c], xj[c], acc);
        dA[(i0 + r) * ldd + j] = accumulate ? old[r] - acc : -acc;
    }
}

}  // namespace

int32_t solve_adjoint_f64(Ctx* ctx, cudaStream_t st, const double* LU, int64_t ld, int64_t n, const int32_t* perm,
                          const double* X, int64_t ldx, const double* G, int64_t ldg, int64_t nrhs, double* Lam,
                          int64_t ldl, double* dA, int64_t ldd, int op, double* Y, int64_t ldy) {
    if (n <= 0 || nrhs <= 0) return B2M_OK;
    // Y = G; Y <- U^{-T} Y; Y <- L^{-T} Y; Lambda = P^T Y
    B2M_TRY(copy_matrix(ctx, st, Y, ldy * 8, G, ldg * 8, n, nrhs));
    B2M_TRY(tri_solve2_f64(ctx, st, LU, ld, n, kTriUt, kTriLt, Y, ldy, nrhs));
    scatter_rows_kernel<<<(unsigned)ceil_div(n * nrhs, 256), 256, 0, st>>>(Lam, ldl, Y, ldy, perm, n, nrhs,
                                                                            ctx->d_status);
    B2M_LAUNCHED(ctx);
    if (!dA) return B2M_OK;
    for (int64_t c0 = 0; c0 < nrhs; c0 += kRkK) {
        const int kc = (int)std::min<int64_t>(kRkK, nrhs - c0);
        const int acc = (op == B2M_DO_ADD || c0 > 0) ? 1 : 0;
        dim3 grid((unsigned)ceil_div(n, kRkCols), (unsigned)ceil_div(n, kRkRows));
        prof_begin(ctx, st, kClsOther);
        if (kc == 1)
            rank_update_kernel<1><<<grid, kRkCols, 0, st>>>(dA, ldd, Lam, ldl, X, ldx, n, (int)c0, kc, acc);
        else if (kc <= 4)
            rank_update_kernel<4><<<grid, kRkCols, 0, st>>>(dA, ldd, Lam, ldl, X, ldx, n, (int)c0, kc, acc);
        else
            rank_update_kernel<kRkK><<<grid, kRkCols, 0, st>>>(dA, ldd, Lam, ldl, X, ldx, n, (int)c0, kc, acc);
        prof_end(ctx, st, kClsOther, 8.0 * n * n * (acc ? 2 : 1) + 16.0 * n * kc);  // bytes: dA once
        B2M_LAUNCHED(ctx);
    }
    return B2M_OK;
}

}  // namespace b2m
