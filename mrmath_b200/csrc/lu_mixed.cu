// lu_mixed.cu -- mixed-precision LU solve: FP32 factorisation whose trailing updates and
// triangular-solve updates run on the tcgen05 tensor cores (TF32 or 3xTF32), FP64 iterative
// refinement (residual b - Ax, update x += d, normwise backward-error stopping test, all in FP64),
// and a plain FP64 re-factorisation when refinement stalls or the FP32 factorisation is singular.
//
// There is no counterpart in the reference (MatrixLinEQSolve, LinAlgLU.pas:481-592, refines a
// fixed number of times in FP64 around an FP64 factorisation); the result is judged against the
// FP64 oracle through its backward error.
#include <cmath>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace b2m {
namespace {

// ------------------------------------------------------------------ small kernels
__global__ void f64_to_f32_kernel(const double* src, int64_t lds, float* dst, int64_t ldd, int64_t rows, int64_t cols) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= rows * cols) return;
    const int64_t r = e / cols, c = e - r * cols;
    dst[r * ldd + c] = (float)src[r * lds + c];
}

__global__ void add_f32_to_f64_kernel(double* x, int64_t ldx, const float* d, int64_t ldd, int64_t rows, int64_t cols) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= rows * cols) return;
    const int64_t r = e / cols, c = e - r * cols;
    x[r * ldx + c] += (double)d[r * ldd + c];
}

// ||A||_inf: max row sum of |a_ij| (one warp per row, then a global max on the bit pattern)
__global__ void norm_inf_kernel(const double* A, int64_t lda, int64_t n, unsigned long long* out) {
    const int64_t row = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    double s = 0.0;
    for (int64_t j = lane; j < n; j += 32) s += fabs(A[row * lda + j]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) atomicMax(out, (unsigned long long)__double_as_longlong(s));
}

// column-wise max |.| of R, X, B (n x k): out[0..k) = |r|, [k..2k) = |x|, [2k..3k) = |b| (bit patterns)
__global__ void colmax3_kernel(const double* R, int64_t ldr, const double* X, int64_t ldx, const double* B, int64_t ldb,
                               int64_t n, int64_t k, unsigned long long* out) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * k) return;
    const int64_t i = e / k, c = e - i * k;
    atomicMax(&out[c], (unsigned long long)__double_as_longlong(fabs(R[i * ldr + c])));
    atomicMax(&out[k + c], (unsigned long long)__double_as_longlong(fabs(X[i * ldx + c])));
    atomicMax(&out[2 * k + c], (unsigned long long)__double_as_longlong(fabs(B[i * ldb + c])));
}

// X[i][:] = B[perm[i]][:] (FP32)
__global__ void gather_rows_f32_kernel(float* X, int64_t ldx, const float* B, int64_t ldb, const int32_t* perm,
                                       int64_t n, int64_t nrhs) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * nrhs) return;
    const int64_t i = e / nrhs, c = e - i * nrhs;
    X[i * ldx + c] = B[(int64_t)perm[i] * ldb + c];
}

__global__ void iota32_kernel(int32_t* v, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = (int32_t)i;
}

unsigned gsz(int64_t n, int b = 256) { return (unsigned)ceil_div(std::max<int64_t>(n, 1), b); }

// ------------------------------------------------------------------ FP32 GEMM through the tensor cores
struct Split {
    float* ah;
    float* al;
    float* bh;
    float* bl;
    int64_t cap;  // floats available in each buffer
    int mode;     // 1 TF32, 3 3xTF32
};

// C(M x N) op= A(M x K) * B(K x N): A is a block of a row-major FP32 matrix (K-major as stored), B a
// row-major block (transposed into Bt for the K-major B operand, and split for 3xTF32).
int32_t f32_gemm(Ctx* ctx, cudaStream_t st, const float* A, int64_t lda, int64_t a_rows, int64_t a_cols, int64_t ar0,
                 int64_t ac0, const float* B, int64_t ldb, int64_t br0, int64_t bc0, float* C, int64_t ldc, int64_t M,
                 int64_t N, int64_t K, int op, const Split& sp) {
    if (M <= 0 || N <= 0 || K <= 0) return B2M_OK;
    const int64_t ldk = round_up(K, 4);
    if (N * ldk > sp.cap || (sp.mode == 3 && M * ldk > sp.cap))
        return fail(ctx, B2M_ERR_UNSUPPORTED, "mixed GEMM scratch too small");
    B2M_TRY(tf32_split(ctx, st, B + br0 * ldb + bc0, ldb, K, N, sp.bh, sp.mode == 3 ? sp.bl : nullptr, ldk, true));
    FOperand bh{sp.bh, ldk, N, K, 0, 0};
    if (sp.mode == 3) {
        B2M_TRY(tf32_split(ctx, st, A + ar0 * lda + ac0, lda, M, K, sp.ah, sp.al, ldk, false));
        FOperand ah{sp.ah, ldk, M, K, 0, 0};
        return sgemm_tc(ctx, st, ah, sp.al, bh, sp.bl, C, ldc, M, N, K, op, 3, true);
    }
    FOperand ah{A, lda, a_rows, a_cols, ar0, ac0};
    return sgemm_tc(ctx, st, ah, nullptr, bh, nullptr, C, ldc, M, N, K, op, 1, true);
}

// triangle of the FP32 LU at (A, lda, n x n), right-hand sides rows of (B, ldb) at column bc0
struct TriF {
    const float* A;
    int64_t lda, n;
    float* B;
    int64_t ldb, bc0, ncols;
};

int32_t trsm_lower_f32(Ctx* ctx, cudaStream_t st, const TriF& t, int64_t r0, int64_t br0, int64_t k, const Split& sp) {
    if (k <= 32)
        return launch_trsm_small<float>(ctx, st, t.A + r0 * t.lda + r0, t.lda, t.B + br0 * t.ldb + t.bc0, t.ldb,
                                        (int)k, (int)t.ncols, false);
    const int64_t k1 = round_up((k + 1) / 2, 32), k2 = k - k1;
    B2M_TRY(trsm_lower_f32(ctx, st, t, r0, br0, k1, sp));
    B2M_TRY(f32_gemm(ctx, st, t.A, t.lda, t.n, t.n, r0 + k1, r0, t.B, t.ldb, br0, t.bc0,
                     t.B + (br0 + k1) * t.ldb + t.bc0, t.ldb, k2, t.ncols, k1, B2M_DO_SUB, sp));
    return trsm_lower_f32(ctx, st, t, r0 + k1, br0 + k1, k2, sp);
}

int32_t trsm_upper_f32(Ctx* ctx, cudaStream_t st, const TriF& t, int64_t r0, int64_t br0, int64_t k, const Split& sp) {
    if (k <= 32)
        return launch_trsm_small<float>(ctx, st, t.A + r0 * t.lda + r0, t.lda, t.B + br0 * t.ldb + t.bc0, t.ldb,
                                        (int)k, (int)t.ncols, true);
    const int64_t k1 = round_up((k + 1) / 2, 32), k2 = k - k1;
    B2M_TRY(trsm_upper_f32(ctx, st, t, r0 + k1, br0 + k1, k2, sp));
    B2M_TRY(f32_gemm(ctx, st, t.A, t.lda, t.n, t.n, r0, r0 + k1, t.B, t.ldb, br0 + k1, t.bc0, t.B + br0 * t.ldb + t.bc0,
                     t.ldb, k1, t.ncols, k2, B2M_DO_SUB, sp));
    return trsm_upper_f32(ctx, st, t, r0, br0, k1, sp);
}

int32_t lu_rec_f32(Ctx* ctx, cudaStream_t st, float* A, int64_t ld, int64_t n, int64_t c0, int64_t width, int32_t* ipiv,
                   int32_t* perm, const Split& sp) {
    if (width <= 32) {
        B2M_TRY(launch_panel<float>(ctx, st, A + c0 * ld + c0, ld, (int)(n - c0), (int)width, (int)c0, (int)c0, ipiv));
        return launch_swaps<float>(ctx, st, A, ld, (int)n, (int)c0, (int)width, ipiv, perm);
    }
    const int64_t nleft = round_up((width + 1) / 2, 32), nright = width - nleft;
    B2M_TRY(lu_rec_f32(ctx, st, A, ld, n, c0, nleft, ipiv, perm, sp));
    TriF t{A, ld, n, A, ld, c0 + nleft, nright};
    B2M_TRY(trsm_lower_f32(ctx, st, t, c0, c0, nleft, sp));
    const int64_t r1 = c0 + nleft;
    B2M_TRY(f32_gemm(ctx, st, A, ld, n, n, r1, c0, A, ld, c0, r1, A + r1 * ld + r1, ld, n - r1, nright, nleft,
                     B2M_DO_SUB, sp));
    return lu_rec_f32(ctx, st, A, ld, n, r1, nright, ipiv, perm, sp);
}

}  // namespace

// FP32 LU with tensor-core updates (graph-captured like the FP64 one)
int32_t lu_factor_f32(Ctx* ctx, cudaStream_t st, float* A, int64_t ld, int64_t n, int32_t* ipiv, int32_t* perm,
                      int mode, float* scratch, int64_t scratch_cap) {
    if (n <= 0) return B2M_OK;
    if ((ld & 3) || !aligned16(A)) return fail(ctx, B2M_ERR_DIM, "lu_factor_f32: ld must be a multiple of 4");
    if (n > panel_max_rows(false, 32)) return fail(ctx, B2M_ERR_UNSUPPORTED, "mixed LU supports n <= 16384");
    Split sp{scratch, scratch + scratch_cap, scratch + 2 * scratch_cap, scratch + 3 * scratch_cap, scratch_cap, mode};
    const GraphKey key{3 + mode * 10, A, ipiv, perm, scratch, ld, n, scratch_cap, 0};
    return run_graph(ctx, st, key, [&](cudaStream_t s) -> int32_t {
        iota32_kernel<<<gsz(n), 256, 0, s>>>(perm, n);
        B2M_LAUNCHED(ctx);
        return lu_rec_f32(ctx, s, A, ld, n, 0, n, ipiv, perm, sp);
    });
}

int32_t lu_solve_f32(Ctx* ctx, cudaStream_t st, const float* LU, int64_t ld, int64_t n, const int32_t* perm, float* B,
                     int64_t ldb, int64_t nrhs, float* tmp, int mode, float* scratch, int64_t scratch_cap) {
    Split sp{scratch, scratch + scratch_cap, scratch + 2 * scratch_cap, scratch + 3 * scratch_cap, scratch_cap, mode};
    const GraphKey key{4 + mode * 10, LU, perm, B, tmp, ld, n, ldb, nrhs};
    return run_graph(ctx, st, key, [&](cudaStream_t s) -> int32_t {
        B2M_CU(ctx, cudaMemcpy2DAsync(tmp, ldb * 4, B, ldb * 4, nrhs * 4, n, cudaMemcpyDeviceToDevice, s));
        gather_rows_f32_kernel<<<gsz(n * nrhs), 256, 0, s>>>(B, ldb, tmp, ldb, perm, n, nrhs);
        B2M_LAUNCHED(ctx);
        TriF t{LU, ld, n, B, ldb, 0, nrhs};
        B2M_TRY(trsm_lower_f32(ctx, s, t, 0, 0, n, sp));
        return trsm_upper_f32(ctx, s, t, 0, 0, n, sp);
    });
}

// ------------------------------------------------------------------ the refinement driver
int32_t solve_mixed(Ctx* ctx, cudaStream_t st, const double* A, int64_t lda, int64_t n, const double* B, int64_t ldb,
                    double* X, int64_t ldx, int64_t nrhs, int mode, int max_iter, double tol, MixedReport* rep) {
    if (mode != 1 && mode != 3) return fail(ctx, B2M_ERR_ARG, "mode must be 1 (TF32) or 3 (3xTF32)");
    if ((lda & 1) || (ldb & 1) || (ldx & 1) || !aligned16(A) || !aligned16(B) || !aligned16(X))
        return fail(ctx, B2M_ERR_DIM, "solve_mixed: device operands need even strides and 16-byte alignment");
    const int64_t ld32 = round_up(n, 32);
    const int64_t ldr = round_up(nrhs, 4);
    const int64_t cap = round_up(n, 32) * (round_up(n, 32) / 2 + 32);
    // workspace layout: [A32 | split scratch x4] in kWsMatD, [r64] kWsF, [r32 | tmp32] kWsE, pivots kWsPiv,
    // norms kWsSmall
    void *pD, *pF, *pE, *pP, *pS;
    B2M_TRY(ws_get(ctx, kWsMatD, (size_t)(n * ld32 + 4 * cap) * sizeof(float), &pD));
    B2M_TRY(ws_get(ctx, kWsF, (size_t)(n * ldr) * sizeof(double), &pF));
    B2M_TRY(ws_get(ctx, kWsE, (size_t)(2 * n * ldr) * sizeof(float), &pE));
    B2M_TRY(ws_get(ctx, kWsPiv, (size_t)(2 * n) * sizeof(int32_t), &pP));
    B2M_TRY(ws_get(ctx, kWsSmall, (size_t)(4 + 3 * nrhs) * sizeof(unsigned long long), &pS));
    float* A32 = (float*)pD;
    float* scratch = A32 + n * ld32;
    double* R = (double*)pF;
    float* r32 = (float*)pE;
    float* t32 = r32 + n * ldr;
    int32_t* ipiv = (int32_t*)pP;
    int32_t* perm = ipiv + n;
    unsigned long long* nrm = (unsigned long long*)pS;
    std::vector<unsigned long long> h((size_t)(1 + 3 * nrhs));

    MixedReport local{};
    if (!rep) rep = &local;
    *rep = MixedReport{};

    B2M_CU(ctx, cudaMemsetAsync(ctx->d_status, 0, kNumStatus * sizeof(int32_t), st));
    f64_to_f32_kernel<<<gsz(n * n), 256, 0, st>>>(A, lda, A32, ld32, n, n);
    B2M_LAUNCHED(ctx);
    B2M_TRY(lu_factor_f32(ctx, st, A32, ld32, n, ipiv, perm, mode, scratch, cap));
    B2M_CU(ctx, cudaMemsetAsync(nrm, 0, sizeof(unsigned long long), st));
    norm_inf_kernel<<<gsz(n, 8), 256, 0, st>>>(A, lda, n, nrm);
    B2M_LAUNCHED(ctx);
    B2M_CU(ctx, cudaMemcpyAsync(ctx->h_status, ctx->d_status, kNumStatus * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    B2M_CU(ctx, cudaMemcpyAsync(h.data(), nrm, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    B2M_CU(ctx, cudaStreamSynchronize(st));
    if (ctx->h_status[kTimeout]) return fail(ctx, B2M_ERR_TIMEOUT, "bounded wait gave up (site %d)", ctx->h_status[kTimeout]);
    const double normA = __builtin_bit_cast(double, h[0]);

    bool converged = false;
    if (ctx->h_status[kInfo] == 0) {
        // x = 0, r = b
        B2M_CU(ctx, cudaMemset2DAsync(X, ldx * 8, 0, nrhs * 8, n, st));
        B2M_TRY(copy_matrix(ctx, st, R, ldr * 8, B, ldb * 8, n, nrhs));
        double prev = INFINITY;
        for (int it = 0; it < max_iter; ++it) {
            // d = (LU)^{-1} P r in FP32, x += d
            f64_to_f32_kernel<<<gsz(n * nrhs), 256, 0, st>>>(R, ldr, r32, ldr, n, nrhs);
            B2M_LAUNCHED(ctx);
            B2M_TRY(lu_solve_f32(ctx, st, A32, ld32, n, perm, r32, ldr, nrhs, t32, mode, scratch, cap));
            add_f32_to_f64_kernel<<<gsz(n * nrhs), 256, 0, st>>>(X, ldx, r32, ldr, n, nrhs);
            B2M_LAUNCHED(ctx);
            // r = b - A x in FP64
            B2M_TRY(copy_matrix(ctx, st, R, ldr * 8, B, ldb * 8, n, nrhs));
            DOperand a{A, lda, n, n, 0, 0, true};
            DOperand b{X, ldx, n, nrhs, 0, 0, false};
            B2M_TRY(dgemm_tiled(ctx, st, a, b, R, ldr, n, nrhs, n, B2M_DO_SUB, false));
            // normwise backward error per column
            B2M_CU(ctx, cudaMemsetAsync(nrm + 1, 0, 3 * nrhs * sizeof(unsigned long long), st));
            colmax3_kernel<<<gsz(n * nrhs), 256, 0, st>>>(R, ldr, X, ldx, B, ldb, n, nrhs, nrm + 1);
            B2M_LAUNCHED(ctx);
            B2M_CU(ctx, cudaMemcpyAsync(h.data() + 1, nrm + 1, 3 * nrhs * sizeof(unsigned long long),
                                        cudaMemcpyDeviceToHost, st));
            B2M_CU(ctx, cudaStreamSynchronize(st));
            double eta = 0.0;
            for (int64_t c = 0; c < nrhs; ++c) {
                const double rn = __builtin_bit_cast(double, h[1 + c]);
                const double xn = __builtin_bit_cast(double, h[1 + nrhs + c]);
                const double bn = __builtin_bit_cast(double, h[1 + 2 * nrhs + c]);
                const double den = normA * xn + bn;
                eta = std::max(eta, den > 0 ? rn / den : (rn > 0 ? INFINITY : 0.0));
            }
            rep->iterations = it + 1;
            rep->backward_error = eta;
            rep->ir_backward_error = eta;
            if (std::isfinite(eta) && eta <= tol) {
                converged = true;
                break;
            }
            // stall: less than a 2x reduction after the second step, or growth
            if (!std::isfinite(eta) || (it >= 1 && eta > 0.5 * prev)) break;
            prev = eta;
        }
    }
    if (converged) return B2M_OK;
    // plain FP64 LU solve on the GPU
    rep->fell_back = 1;
    return solve_plain_f64(ctx, st, A, lda, n, B, ldb, X, ldx, nrhs, rep);
}

int32_t solve_plain_f64(Ctx* ctx, cudaStream_t st, const double* A, int64_t lda, int64_t n, const double* B,
                        int64_t ldb, double* X, int64_t ldx, int64_t nrhs, MixedReport* rep) {
    const int64_t ld = round_up(n, 16);
    void *pC, *pP, *pS;
    B2M_TRY(ws_get(ctx, kWsMatC, (size_t)(n * ld) * sizeof(double), &pC));
    B2M_TRY(ws_get(ctx, kWsPiv, (size_t)(2 * n) * sizeof(int32_t), &pP));
    B2M_TRY(ws_get(ctx, kWsSmall, (size_t)(4 + 3 * nrhs) * sizeof(unsigned long long), &pS));
    double* LU = (double*)pC;
    int32_t* ipiv = (int32_t*)pP;
    B2M_TRY(copy_matrix(ctx, st, LU, ld * 8, A, lda * 8, n, n));
    B2M_CU(ctx, cudaMemsetAsync(ctx->d_status, 0, kNumStatus * sizeof(int32_t), st));
    B2M_TRY(lu_factor_f64(ctx, st, LU, ld, n, ipiv, ipiv + n));
    B2M_TRY(copy_matrix(ctx, st, X, ldx * 8, B, ldb * 8, n, nrhs));
    B2M_TRY(lu_solve_f64(ctx, st, LU, ld, n, ipiv + n, X, ldx, nrhs));
    B2M_CU(ctx, cudaMemcpyAsync(ctx->h_status, ctx->d_status, kNumStatus * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    B2M_CU(ctx, cudaStreamSynchronize(st));
    if (ctx->h_status[kTimeout]) return fail(ctx, B2M_ERR_TIMEOUT, "bounded wait gave up (site %d)", ctx->h_status[kTimeout]);
    if (ctx->h_status[kInfo]) return B2M_SINGULAR;
    if (rep) {
        // backward error of the FP64 solution, for the report
        void* pF;
        const int64_t ldr = round_up(nrhs, 4);
        B2M_TRY(ws_get(ctx, kWsF, (size_t)(n * ldr) * sizeof(double), &pF));
        double* R = (double*)pF;
        unsigned long long* nrm = (unsigned long long*)pS;
        B2M_TRY(copy_matrix(ctx, st, R, ldr * 8, B, ldb * 8, n, nrhs));
        DOperand a{A, lda, n, n, 0, 0, true};
        DOperand b{X, ldx, n, nrhs, 0, 0, false};
        B2M_TRY(dgemm_tiled(ctx, st, a, b, R, ldr, n, nrhs, n, B2M_DO_SUB, false));
        B2M_CU(ctx, cudaMemsetAsync(nrm, 0, (1 + 3 * nrhs) * sizeof(unsigned long long), st));
        norm_inf_kernel<<<gsz(n, 8), 256, 0, st>>>(A, lda, n, nrm);
        B2M_LAUNCHED(ctx);
        colmax3_kernel<<<gsz(n * nrhs), 256, 0, st>>>(R, ldr, X, ldx, B, ldb, n, nrhs, nrm + 1);
        B2M_LAUNCHED(ctx);
        std::vector<unsigned long long> h((size_t)(1 + 3 * nrhs));
        B2M_CU(ctx, cudaMemcpyAsync(h.data(), nrm, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        B2M_CU(ctx, cudaStreamSynchronize(st));
        const double normA = __builtin_bit_cast(double, h[0]);
        double eta = 0.0;
        for (int64_t c = 0; c < nrhs; ++c) {
            const double den = normA * __builtin_bit_cast(double, h[1 + nrhs + c]) +
                               __builtin_bit_cast(double, h[1 + 2 * nrhs + c]);
            const double rn = __builtin_bit_cast(double, h[1 + c]);
            eta = std::max(eta, den > 0 ? rn / den : 0.0);
        }
        rep->backward_error = eta;
    }
    return B2M_OK;
}

}  // namespace b2m
