// chol.cu -- Cholesky factorisation A = L L^T of a symmetric positive-definite FP64 matrix and the
// solve built on it (the next dense factorisation on the LU path's DGEMM and triangular sweeps).
//
// Reference: TDoubleMatrix.Cholesky (DblMatrix.pas:967-990) -> MatrixCholeskyInPlace4
// (LinAlgCholesky.pas:106-123), a left-looking blocked Cholesky with 32-column panels
// (InternalBlkCholeskyInPlace :54-103: rank-k update of the diagonal block, unblocked factorisation
// MatrixCholeskyInPlace2 :205-250, MultT2 update of the column below, triangular solve with the
// reciprocal of each diagonal element); the Numerical-Recipes form MatrixCholeskyInPlace (:270-332,
// L below the diagonal, its diagonal in a separate vector P) and MatrixCholeskySolveLinEq
// (:352-421).  Result: 0 = crOk, 1 = crNoPositiveDefinite (MatrixConst.pas:30) when a diagonal
// element is <= 0 or NaN before its square root.
//
// B200 design: outer panels of 256 columns; inside a panel, 32-column leaves are updated
// left-looking by one DMMA GEMM each (the leaf's rows times the panel's earlier columns, K <= 224),
// then factored by chol_leaf_kernel: every CTA factors the leaf's 32 x 32 diagonal block itself
// (one warp, lane = row, shuffles; no grid-wide wait) and solves its 128 rows of the block column,
// x L11^T = a, by substitution with L11 in shared memory.  After a panel, the trailing lower
// triangle is updated by DMMA GEMMs in four column slabs (about 1.25x the triangle's flops).  The
// factorisation runs on a workspace copy, so the caller's strict upper triangle is never written.
#include <cfloat>

#include "common.cuh"
#include "kernels.cuh"

namespace b2m {
namespace {

constexpr int kChLeaf = 32;        // leaf width
constexpr int kChPanel = 256;      // outer panel width
constexpr int kChRows = 128;       // rows per leaf CTA
constexpr int kChSlabs = 4;        // column slabs of a trailing update

// Leaf [c, c + w) of the n x n matrix (row stride ld), w <= 32: its columns are up to date.
// Grid: ceil((n - c) / 128) CTAs of 128 threads; thread t of CTA b owns row c + 128 b + t.
__global__ void __launch_bounds__(kChRows) chol_leaf_kernel(double* A, int64_t ld, int n, int c, int w,
                                                            int32_t* status) {
    __shared__ double s_l[kChLeaf][kChLeaf + 1];  // factored diagonal block, s_l[i][k] = L(c+i, c+k)
    __shared__ int s_bad;
    if (status[kInfo] != 0) return;
    const int t = threadIdx.x, lane = t & 31;
    if (t == 0) s_bad = 0;
    if (t < 32) {
        // lane i holds row i of the diagonal block (lower part), right-looking factorisation
        double r[kChLeaf];
        const double* arow = A + (int64_t)(c + min(lane, w - 1)) * ld + c;
#pragma unroll
        for (int k = 0; k < kChLeaf; ++k) r[k] = (lane < w && k < w && k <= lane) ? arow[k] : 0.0;
        bool bad = false;
#pragma unroll
        for (int j = 0; j < kChLeaf; ++j) {
            if (j < w) {
                const double pj = __shfl_sync(0xffffffffu, r[j], j);
                if (!(pj > 0.0)) {  // <= 0 or NaN: not positive definite (uniform across the warp)
                    bad = true;
                    break;
                }
                const double d = sqrt(pj);
                if (lane == j) r[j] = d;
                if (lane > j) r[j] = r[j] / d;
#pragma unroll
                for (int k = j + 1; k < kChLeaf; ++k) {
                    const double lkj = __shfl_sync(0xffffffffu, r[j], k);  // L(k, j) from lane k
                    if (k < w && lane >= k) r[k] = fma(-r[j], lkj, r[k]);
                }
            }
        }
        if (bad) {
            if (lane == 0) {
                s_bad = 1;
                if (blockIdx.x == 0) atomicExch(&status[kInfo], 1);
            }
        } else {
#pragma unroll
            for (int k = 0; k < kChLeaf; ++k) s_l[lane][k] = r[k];
        }
    }
    __syncthreads();
    if (s_bad) return;
    const int row = c + blockIdx.x * kChRows + t;
    if (row >= n) return;
    double* a = A + (int64_t)row * ld + c;
    if (row < c + w) {  // the diagonal block's own rows: lower part only
        const int i = row - c;
        for (int k = 0; k <= i; ++k) a[k] = s_l[i][k];
        return;
    }
    // x L11^T = a: x_j = (a_j - sum_{k<j} x_k L(j, k)) / L(j, j)
    double x[kChLeaf];
#pragma unroll
    for (int k = 0; k < kChLeaf; ++k) x[k] = k < w ? a[k] : 0.0;
#pragma unroll
    for (int j = 0; j < kChLeaf; ++j) {
        if (j < w) {
            double s = x[j];
#pragma unroll
            for (int k = 0; k < j; ++k) s = fma(-x[k], s_l[j][k], s);
            x[j] = s / s_l[j][j];
        }
    }
#pragma unroll
    for (int k = 0; k < kChLeaf; ++k)
        if (k < w) a[k] = x[k];
}

// dst's lower triangle (diagonal included) <- src's, when status[kInfo] == 0
__global__ void copy_lower_kernel(double* dst, int64_t ldd, const double* src, int64_t lds, int64_t n,
                                  const int32_t* status) {
    if (status && status[kInfo] != 0) return;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * n) return;
    const int64_t i = e / n, j = e - i * n;
    if (j <= i) dst[i * ldd + j] = src[i * lds + j];
}

// X's strict upper triangle <- the transpose of its strict lower triangle (U = L^T next to L)
__global__ void mirror_lower_kernel(double* X, int64_t ld, int64_t n) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * n) return;
    const int64_t i = e / n, j = e - i * n;
    if (j > i) X[i * ld + j] = X[j * ld + i];
}

// L's strict lower triangle and P's diagonal from one factor (NR form): Lnr[i][j] = F[i][j] (j < i),
// P[i] = F[i][i] (P element i at byte offset i * lwp)
__global__ void split_nr_kernel(double* Lnr, int64_t ldl, double* P, int64_t lwp, const double* F, int64_t ldf,
                                int64_t n, const int32_t* status) {
    if (status[kInfo] != 0) return;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * n) return;
    const int64_t i = e / n, j = e - i * n;
    if (j < i) Lnr[i * ldl + j] = F[i * ldf + j];
    if (j == i) *reinterpret_cast<double*>(reinterpret_cast<char*>(P) + i * lwp) = F[i * ldf + i];
}

// F <- Lnr's strict lower triangle with P on the diagonal (the NR form joined into one factor)
__global__ void join_nr_kernel(double* F, int64_t ldf, const double* Lnr, int64_t ldl, const double* P, int64_t lwp,
                               int64_t n) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * n) return;
    const int64_t i = e / n, j = e - i * n;
    if (j < i) F[i * ldf + j] = Lnr[i * ldl + j];
    if (j == i) F[i * ldf + i] = *reinterpret_cast<const double*>(reinterpret_cast<const char*>(P) + i * lwp);
}

unsigned blocks_for(int64_t e) { return (unsigned)ceil_div(std::max<int64_t>(e, 1), 256); }

}  // namespace

int32_t chol_factor_f64(Ctx* ctx, cudaStream_t st, double* A, int64_t ld, int64_t n) {
    if (n <= 0) return B2M_OK;
    if ((ld & 1) || !aligned16(A)) return fail(ctx, B2M_ERR_DIM, "chol_factor_f64: ld must be even, A 16-byte aligned");
    if (n > (1 << 30)) return fail(ctx, B2M_ERR_UNSUPPORTED, "chol_factor_f64: n too large");
    const GraphKey key{20, A, nullptr, nullptr, ctx->d_status, ld, n, 0, 0};
    return run_graph(ctx, st, key, [&](cudaStream_t s) -> int32_t {
        for (int64_t k0 = 0; k0 < n; k0 += kChPanel) {
            const int64_t k1 = std::min(n, k0 + kChPanel);
            for (int64_t c = k0; c < k1; c += kChLeaf) {
                const int64_t w = std::min<int64_t>(kChLeaf, k1 - c);
                if (c > k0) {  // left-looking: A[c:n, c:c+w] -= L[c:n, k0:c] L[c:c+w, k0:c]^T
                    DOperand a{A, ld, n, n, c, k0, true};
                    DOperand b{A, ld, n, n, c, k0, true};
                    B2M_TRY(dgemm_tiled(ctx, s, a, b, A + c * ld + c, ld, n - c, w, c - k0, B2M_DO_SUB, true));
                }
                prof_begin(ctx, s, kClsPanel);
                chol_leaf_kernel<<<(unsigned)ceil_div(n - c, kChRows), kChRows, 0, s>>>(A, ld, (int)n, (int)c, (int)w,
                                                                                      ctx->d_status);
                prof_end(ctx, s, kClsPanel, 2.0 * (n - c) * w * 8.0);
                B2M_LAUNCHED(ctx);
            }
            // trailing lower triangle: slabs of columns [cs, ce): rows [cs, n) -= L[cs:n, k0:k1] L[cs:ce, k0:k1]^T
            const int64_t m = n - k1;
            if (m <= 0) continue;
            const int64_t slab = round_up(ceil_div(m, kChSlabs), 128);
            for (int64_t cs = k1; cs < n; cs += slab) {
                const int64_t ce = std::min(n, cs + slab);
                DOperand a{A, ld, n, n, cs, k0, true};
                DOperand b{A, ld, n, n, cs, k0, true};
                B2M_TRY(dgemm_tiled(ctx, s, a, b, A + cs * ld + cs, ld, n - cs, ce - cs, k1 - k0, B2M_DO_SUB, true));
            }
        }
        return B2M_OK;
    });
}

// Solves A X = B from a Cholesky factor F (lower triangle, diagonal included, row stride ldf):
// the factor is copied into the workspace W (n x ldw), mirrored so that U = L^T sits above the
// diagonal, then two FP64 sweeps: L y = b (the transposed upper triangle, true division) and
// L^T x = y.  B (n x nrhs, ldb) is overwritten with X.
int32_t chol_solve_f64(Ctx* ctx, cudaStream_t st, const double* F, int64_t ldf, int64_t n, double* W, int64_t ldw,
                       double* B, int64_t ldb, int64_t nrhs) {
    if (n <= 0 || nrhs <= 0) return B2M_OK;
    B2M_CU(ctx, cudaMemcpy2DAsync(W, ldw * 8, F, ldf * 8, n * 8, n, cudaMemcpyDeviceToDevice, st));
    mirror_lower_kernel<<<blocks_for(n * n), 256, 0, st>>>(W, ldw, n);
    B2M_LAUNCHED(ctx);
    return tri_solve2_f64(ctx, st, W, ldw, n, kTriUt, kTriU, B, ldb, nrhs);
}

int32_t copy_lower(Ctx* ctx, cudaStream_t st, double* dst, int64_t ldd, const double* src, int64_t lds, int64_t n,
                   bool only_if_ok) {
    if (n <= 0) return B2M_OK;
    copy_lower_kernel<<<blocks_for(n * n), 256, 0, st>>>(dst, ldd, src, lds, n, only_if_ok ? ctx->d_status : nullptr);
    B2M_LAUNCHED(ctx);
    return B2M_OK;
}

int32_t split_nr(Ctx* ctx, cudaStream_t st, double* Lnr, int64_t ldl, double* P, int64_t lwp, const double* F,
                 int64_t ldf, int64_t n) {
    if (n <= 0) return B2M_OK;
    split_nr_kernel<<<blocks_for(n * n), 256, 0, st>>>(Lnr, ldl, P, lwp, F, ldf, n, ctx->d_status);
    B2M_LAUNCHED(ctx);
    return B2M_OK;
}

int32_t join_nr(Ctx* ctx, cudaStream_t st, double* F, int64_t ldf, const double* Lnr, int64_t ldl, const double* P,
                int64_t lwp, int64_t n) {
    if (n <= 0) return B2M_OK;
    join_nr_kernel<<<blocks_for(n * n), 256, 0, st>>>(F, ldf, Lnr, ldl, P, lwp, n);
    B2M_LAUNCHED(ctx);
    return B2M_OK;
}

}  // namespace b2m
