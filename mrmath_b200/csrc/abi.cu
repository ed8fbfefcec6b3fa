// abi.cu -- the extern "C" entry points of b2m.h for GEMM, LU, back-substitution, inverse,
// determinant and the linear-equation solve (plain FP64 form).
//
// Host-buffer calls (b2m_Matrix*) mirror the reference routines of the same name: they copy
// the operands into library-owned device buffers whose row stride is padded for TMA, run the
// device path on the context stream, copy the results back and return the reference's result
// code.  Device-buffer calls (b2m_dev_*) run asynchronously on the context stream.
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "kernels.cuh"

using namespace b2m;

namespace {

Ctx* as_ctx(b2m_ctx* h) { return reinterpret_cast<Ctx*>(h); }

int64_t padded_ld(int64_t cols) { return round_up(std::max<int64_t>(cols, 1), 16); }

// the reference asserts LineWidth >= width*sizeof(double); strides must also be whole doubles
bool lw_ok(int64_t lw, int64_t cols) { return lw >= cols * 8 && (lw % 8) == 0; }

int32_t upload(Ctx* ctx, double* dst, int64_t ld, const double* src, int64_t lw_bytes, int64_t rows, int64_t cols) {
    if (rows <= 0 || cols <= 0) return B2M_OK;
    B2M_CU(ctx, cudaMemcpy2DAsync(dst, ld * 8, src, lw_bytes, cols * 8, rows, cudaMemcpyHostToDevice, ctx->stream));
    return B2M_OK;
}
int32_t download(Ctx* ctx, double* dst, int64_t lw_bytes, const double* src, int64_t ld, int64_t rows, int64_t cols) {
    if (rows <= 0 || cols <= 0) return B2M_OK;
    B2M_CU(ctx, cudaMemcpy2DAsync(dst, lw_bytes, src, ld * 8, cols * 8, rows, cudaMemcpyDeviceToHost, ctx->stream));
    return B2M_OK;
}

int32_t reset_status(Ctx* ctx) {
    B2M_CU(ctx, cudaMemsetAsync(ctx->d_status, 0, kNumStatus * sizeof(int32_t), ctx->stream));
    return B2M_OK;
}

// reads the status words; returns B2M_SINGULAR / B2M_ERR_TIMEOUT / B2M_OK
int32_t finish(Ctx* ctx) {
    B2M_CU(ctx, cudaMemcpyAsync(ctx->h_status, ctx->d_status, kNumStatus * sizeof(int32_t), cudaMemcpyDeviceToHost,
                                ctx->stream));
    B2M_CU(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->h_status[kTimeout] != 0)
        return fail(ctx, B2M_ERR_TIMEOUT, "a bounded device wait gave up (site %d)", ctx->h_status[kTimeout]);
    return ctx->h_status[kInfo] != 0 ? B2M_SINGULAR : B2M_OK;
}

struct MultShape {
    int64_t M, N, K;
};

int32_t mult_shape(Ctx* ctx, int32_t trans, int64_t w1, int64_t h1, int64_t w2, int64_t h2, MultShape* s) {
    if (w1 < 0 || h1 < 0 || w2 < 0 || h2 < 0) return fail(ctx, B2M_ERR_DIM, "negative dimension");
    switch (trans) {
        case 0:
            if (w1 != h2) return fail(ctx, B2M_ERR_DIM, "MatrixMult: width1 (%lld) != height2 (%lld)", (long long)w1,
                                      (long long)h2);
            *s = {h1, w2, w1};
            return B2M_OK;
        case 1:
            if (h1 != h2) return fail(ctx, B2M_ERR_DIM, "MatrixMultT1: height1 != height2");
            *s = {w1, w2, h1};
            return B2M_OK;
        case 2:
            if (w1 != w2) return fail(ctx, B2M_ERR_DIM, "MatrixMultT2: width1 != width2");
            *s = {h1, h2, w1};
            return B2M_OK;
        default: return fail(ctx, B2M_ERR_ARG, "trans must be 0, 1 or 2");
    }
}

// GEMM on device operands that satisfy the TMA rules (16-byte aligned base, even stride)
int32_t mult_device_aligned(Ctx* ctx, int32_t trans, int32_t op, const MultShape& s, const double* A, int64_t lda,
                            int64_t arows, int64_t acols, const double* B, int64_t ldb, int64_t brows, int64_t bcols,
                            double* C, int64_t ldc) {
    DOperand a{A, lda, arows, acols, 0, 0, trans != 1};
    DOperand b{B, ldb, brows, bcols, 0, 0, trans == 2};
    return dgemm_tiled(ctx, ctx->stream, a, b, C, ldc, s.M, s.N, s.K, op, false);
}

}  // namespace

// ======================================================================================= GEMM
extern "C" int32_t b2m_MatrixMultEx(b2m_ctx* h, double* dest, int64_t destLineWidth, const double* mt1,
                                    const double* mt2, int64_t width1, int64_t height1, int64_t width2,
                                    int64_t height2, int64_t LineWidth1, int64_t LineWidth2, int32_t op,
                                    int32_t trans) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!dest || !mt1 || !mt2) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (op < 0 || op > 2) return fail(ctx, B2M_ERR_ARG, "op must be 0 (doNone), 1 (doAdd) or 2 (doSub)");
    MultShape s;
    B2M_TRY(mult_shape(ctx, trans, width1, height1, width2, height2, &s));
    if (!lw_ok(LineWidth1, width1) || !lw_ok(LineWidth2, width2) || !lw_ok(destLineWidth, s.N))
        return fail(ctx, B2M_ERR_DIM, "Line widths do not match");
    if (s.M == 0 || s.N == 0) return B2M_OK;
    cudaSetDevice(ctx->device);
    const int64_t lda = padded_ld(width1), ldb = padded_ld(width2), ldc = padded_ld(s.N);
    void *pa, *pb, *pc;
    B2M_TRY(ws_get(ctx, kWsMatA, (size_t)(std::max<int64_t>(height1, 1) * lda * 8), &pa));
    B2M_TRY(ws_get(ctx, kWsMatB, (size_t)(std::max<int64_t>(height2, 1) * ldb * 8), &pb));
    B2M_TRY(ws_get(ctx, kWsMatC, (size_t)(s.M * ldc * 8), &pc));
    double *dA = (double*)pa, *dB = (double*)pb, *dC = (double*)pc;
    B2M_TRY(upload(ctx, dA, lda, mt1, LineWidth1, height1, width1));
    B2M_TRY(upload(ctx, dB, ldb, mt2, LineWidth2, height2, width2));
    if (op != B2M_DO_NONE) B2M_TRY(upload(ctx, dC, ldc, dest, destLineWidth, s.M, s.N));
    B2M_TRY(reset_status(ctx));
    B2M_TRY(mult_device_aligned(ctx, trans, op, s, dA, lda, height1, width1, dB, ldb, height2, width2, dC, ldc));
    B2M_TRY(download(ctx, dest, destLineWidth, dC, ldc, s.M, s.N));
    return finish(ctx);
}

extern "C" int32_t b2m_dev_MatrixMultEx(b2m_ctx* h, double* dest, int64_t destLineWidth, const double* mt1,
                                        const double* mt2, int64_t width1, int64_t height1, int64_t width2,
                                        int64_t height2, int64_t LineWidth1, int64_t LineWidth2, int32_t op,
                                        int32_t trans) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!dest || !mt1 || !mt2) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (op < 0 || op > 2) return fail(ctx, B2M_ERR_ARG, "invalid op");
    MultShape s;
    B2M_TRY(mult_shape(ctx, trans, width1, height1, width2, height2, &s));
    if (!lw_ok(LineWidth1, width1) || !lw_ok(LineWidth2, width2) || !lw_ok(destLineWidth, s.N))
        return fail(ctx, B2M_ERR_DIM, "Line widths do not match");
    if (s.M == 0 || s.N == 0) return B2M_OK;
    const double* A = mt1;
    const double* B = mt2;
    int64_t lda = LineWidth1 / 8, ldb = LineWidth2 / 8;
    // operands that break the TMA rules are repacked into aligned workspaces
    if (!aligned16(A) || (LineWidth1 & 15)) {
        void* p;
        const int64_t ld = padded_ld(width1);
        B2M_TRY(ws_get(ctx, kWsMatA, (size_t)(std::max<int64_t>(height1, 1) * ld * 8), &p));
        B2M_TRY(copy_matrix(ctx, ctx->stream, (double*)p, ld * 8, A, LineWidth1, height1, width1));
        A = (const double*)p;
        lda = ld;
    }
    if (!aligned16(B) || (LineWidth2 & 15)) {
        void* p;
        const int64_t ld = padded_ld(width2);
        B2M_TRY(ws_get(ctx, kWsMatB, (size_t)(std::max<int64_t>(height2, 1) * ld * 8), &p));
        B2M_TRY(copy_matrix(ctx, ctx->stream, (double*)p, ld * 8, B, LineWidth2, height2, width2));
        B = (const double*)p;
        ldb = ld;
    }
    return mult_device_aligned(ctx, trans, op, s, A, lda, height1, width1, B, ldb, height2, width2, dest,
                               destLineWidth / 8);
}

// ======================================================================================= LU
namespace {

// factor the n x n matrix at host A (LineWidthA) into device workspace; leaves LU in kWsMatA
int32_t factor_host(Ctx* ctx, const double* A, int64_t lwA, int64_t n, double** dLU, int64_t* ld, int32_t** dpiv,
                    int32_t** dperm) {
    *ld = padded_ld(n);
    void *pa, *pp;
    B2M_TRY(ws_get(ctx, kWsMatA, (size_t)(n * *ld * 8), &pa));
    B2M_TRY(ws_get(ctx, kWsPiv, (size_t)(2 * n * 4), &pp));
    *dLU = (double*)pa;
    *dpiv = (int32_t*)pp;
    *dperm = *dpiv + n;
    B2M_TRY(upload(ctx, *dLU, *ld, A, lwA, n, n));
    B2M_CU(ctx, cudaMemsetAsync(*dpiv, 0, (size_t)n * 4, ctx->stream));
    B2M_TRY(reset_status(ctx));
    return lu_factor_f64(ctx, ctx->stream, *dLU, *ld, n, *dpiv, *dperm);
}

}  // namespace

extern "C" int32_t b2m_MatrixLUDecomp(b2m_ctx* h, const double* A, int64_t LineWidthA, double* LUDecomp,
                                      int64_t LineWidthLU, int64_t width, int32_t* indx) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!A || !LUDecomp || !indx) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (width <= 0 || !lw_ok(LineWidthA, width) || !lw_ok(LineWidthLU, width))
        return fail(ctx, B2M_ERR_DIM, "Dimension Error");
    cudaSetDevice(ctx->device);
    double* dLU;
    int64_t ld;
    int32_t *dpiv, *dperm;
    std::memset(indx, 0, (size_t)width * sizeof(int32_t));  // FillChar(indx^, ...) LinAlgLU.pas:287
    B2M_TRY(factor_host(ctx, A, LineWidthA, width, &dLU, &ld, &dpiv, &dperm));
    B2M_TRY(download(ctx, LUDecomp, LineWidthLU, dLU, ld, width, width));
    B2M_CU(ctx, cudaMemcpyAsync(indx, dpiv, (size_t)width * 4, cudaMemcpyDeviceToHost, ctx->stream));
    return finish(ctx);
}

extern "C" int32_t b2m_MatrixLUDecompInPlace(b2m_ctx* h, double* A, int64_t LineWidthA, int64_t width,
                                             int32_t* indx) {
    return b2m_MatrixLUDecomp(h, A, LineWidthA, A, LineWidthA, width, indx);
}

extern "C" int32_t b2m_MatrixLUBackSubst(b2m_ctx* h, const double* LUDecomp, int64_t LineWidthLU, int64_t width,
                                         const int32_t* indx, double* B, int64_t LineWidthB, int64_t nrhs) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!LUDecomp || !indx || !B) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (width <= 0 || nrhs <= 0 || !lw_ok(LineWidthLU, width) || !lw_ok(LineWidthB, nrhs))
        return fail(ctx, B2M_ERR_DIM, "Dimension Error");
    cudaSetDevice(ctx->device);
    const int64_t n = width, ld = padded_ld(n), ldb = padded_ld(nrhs);
    void *pa, *pb, *pp;
    B2M_TRY(ws_get(ctx, kWsMatA, (size_t)(n * ld * 8), &pa));
    B2M_TRY(ws_get(ctx, kWsMatB, (size_t)(n * ldb * 8), &pb));
    B2M_TRY(ws_get(ctx, kWsPiv, (size_t)(2 * n * 4), &pp));
    int32_t* dpiv = (int32_t*)pp;
    int32_t* dperm = dpiv + n;
    B2M_TRY(upload(ctx, (double*)pa, ld, LUDecomp, LineWidthLU, n, n));
    B2M_TRY(upload(ctx, (double*)pb, ldb, B, LineWidthB, n, nrhs));
    B2M_CU(ctx, cudaMemcpyAsync(dpiv, indx, (size_t)n * 4, cudaMemcpyHostToDevice, ctx->stream));
    B2M_TRY(reset_status(ctx));
    B2M_TRY(perm_from_ipiv(ctx, ctx->stream, dpiv, n, dperm));
    B2M_TRY(lu_solve_f64(ctx, ctx->stream, (double*)pa, ld, n, dperm, (double*)pb, ldb, nrhs));
    B2M_TRY(download(ctx, B, LineWidthB, (double*)pb, ldb, n, nrhs));
    return finish(ctx);
}

extern "C" int32_t b2m_MatrixInverseInPlace(b2m_ctx* h, double* A, int64_t LineWidthA, int64_t width) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!A) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (width <= 0 || !lw_ok(LineWidthA, width)) return fail(ctx, B2M_ERR_DIM, "Dimension Error");
    cudaSetDevice(ctx->device);
    double* dLU;
    int64_t ld;
    int32_t *dpiv, *dperm;
    B2M_TRY(factor_host(ctx, A, LineWidthA, width, &dLU, &ld, &dpiv, &dperm));
    const int32_t st = finish(ctx);
    if (st != B2M_OK) return st;  // singular: A is left as it was (the reference works on a copy)
    void* pb;
    B2M_TRY(ws_get(ctx, kWsMatB, (size_t)(width * ld * 8), &pb));
    double* X = (double*)pb;
    B2M_CU(ctx, cudaMemset2DAsync(X, ld * 8, 0, width * 8, width, ctx->stream));
    B2M_TRY(set_diagonal(ctx, ctx->stream, X, ld, width, 1.0));
    B2M_TRY(lu_solve_f64(ctx, ctx->stream, dLU, ld, width, dperm, X, ld, width));
    B2M_TRY(download(ctx, A, LineWidthA, X, ld, width, width));
    return finish(ctx);
}

extern "C" int32_t b2m_MatrixDeterminant(b2m_ctx* h, const double* A, int64_t LineWidthA, int64_t width,
                                         double* det) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!A || !det) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (width <= 0 || !lw_ok(LineWidthA, width)) return fail(ctx, B2M_ERR_DIM, "Dimension error");
    cudaSetDevice(ctx->device);
    double* dLU;
    int64_t ld;
    int32_t *dpiv, *dperm;
    B2M_TRY(factor_host(ctx, A, LineWidthA, width, &dLU, &ld, &dpiv, &dperm));
    void* ps;
    B2M_TRY(ws_get(ctx, kWsSmall, 256, &ps));
    B2M_TRY(lu_determinant(ctx, ctx->stream, dLU, ld, width, dpiv, (double*)ps));
    B2M_CU(ctx, cudaMemcpyAsync(det, ps, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    const int32_t st = finish(ctx);
    if (st == B2M_SINGULAR) {
        *det = 0.0;  // MatrixDeterminant returns 0 for a singular matrix
        return B2M_OK;
    }
    return st;
}

namespace {

// X = A^{-1} B with optional fixed-count FP64 refinement; all operands on the device with
// TMA-friendly strides.  dA is overwritten by the factors when keepA == nullptr.
int32_t solve_device(Ctx* ctx, double* dLU, int64_t ld, int64_t n, const double* dAorig, int64_t ldAo,
                     const double* dB, int64_t ldb, double* dX, int64_t ldx, int64_t nrhs, int64_t numRef,
                     int32_t* dpiv, int32_t* dperm) {
    B2M_TRY(lu_factor_f64(ctx, ctx->stream, dLU, ld, n, dpiv, dperm));
    B2M_TRY(copy_matrix(ctx, ctx->stream, dX, ldx * 8, dB, ldb * 8, n, nrhs));
    B2M_TRY(lu_solve_f64(ctx, ctx->stream, dLU, ld, n, dperm, dX, ldx, nrhs));
    if (numRef > 0) {
        void* pr;
        B2M_TRY(ws_get(ctx, kWsF, (size_t)(n * ldx * 8), &pr));
        double* R = (double*)pr;
        for (int64_t it = 0; it < numRef; ++it) {
            // R = B - A X (refinement step of MatrixLinEQSolve :542-586 with the sign folded)
            B2M_TRY(copy_matrix(ctx, ctx->stream, R, ldx * 8, dB, ldb * 8, n, nrhs));
            DOperand a{dAorig, ldAo, n, n, 0, 0, true};
            DOperand b{dX, ldx, n, nrhs, 0, 0, false};
            B2M_TRY(dgemm_tiled(ctx, ctx->stream, a, b, R, ldx, n, nrhs, n, B2M_DO_SUB, true));
            B2M_TRY(lu_solve_f64(ctx, ctx->stream, dLU, ld, n, dperm, R, ldx, nrhs));
            // X += R
            B2M_TRY(axpy_matrix(ctx, ctx->stream, dX, ldx, R, ldx, n, nrhs));
        }
    }
    return B2M_OK;
}

}  // namespace

extern "C" int32_t b2m_MatrixLinEQSolve(b2m_ctx* h, const double* A, int64_t LineWidthA, int64_t width,
                                        const double* B, int64_t LineWidthB, double* X, int64_t LineWidthX,
                                        int64_t Width2, int64_t NumRefinements) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!A || !B || !X) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (width <= 0 || Width2 <= 0 || !lw_ok(LineWidthA, width) || !lw_ok(LineWidthB, Width2) ||
        !lw_ok(LineWidthX, Width2) || NumRefinements < 0)
        return fail(ctx, B2M_ERR_DIM, "Dimension error");
    cudaSetDevice(ctx->device);
    const int64_t n = width, ld = padded_ld(n), ldb = padded_ld(Width2);
    void *pa, *pb, *px, *pp, *pc = nullptr;
    B2M_TRY(ws_get(ctx, kWsMatA, (size_t)(n * ld * 8), &pa));
    B2M_TRY(ws_get(ctx, kWsMatB, (size_t)(n * ldb * 8), &pb));
    B2M_TRY(ws_get(ctx, kWsMatD, (size_t)(n * ldb * 8), &px));
    B2M_TRY(ws_get(ctx, kWsPiv, (size_t)(2 * n * 4), &pp));
    B2M_TRY(upload(ctx, (double*)pa, ld, A, LineWidthA, n, n));
    B2M_TRY(upload(ctx, (double*)pb, ldb, B, LineWidthB, n, Width2));
    if (NumRefinements > 0) {
        B2M_TRY(ws_get(ctx, kWsMatC, (size_t)(n * ld * 8), &pc));
        B2M_TRY(copy_matrix(ctx, ctx->stream, (double*)pc, ld * 8, (double*)pa, ld * 8, n, n));
    }
    B2M_TRY(reset_status(ctx));
    int32_t* dpiv = (int32_t*)pp;
    B2M_TRY(solve_device(ctx, (double*)pa, ld, n, (double*)pc, ld, (double*)pb, ldb, (double*)px, ldb, Width2,
                         NumRefinements, dpiv, dpiv + n));
    const int32_t st = finish(ctx);
    if (st != B2M_OK) return st;  // singular: X untouched, as in the reference
    B2M_TRY(download(ctx, X, LineWidthX, (double*)px, ldb, n, Width2));
    return finish(ctx);
}

// ======================================================================================= device twins
extern "C" int32_t b2m_dev_MatrixLUDecompInPlace(b2m_ctx* h, double* A, int64_t LineWidthA, int64_t width,
                                                 int32_t* indx, int32_t* status) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!A || !indx) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (width <= 0 || !lw_ok(LineWidthA, width)) return fail(ctx, B2M_ERR_DIM, "Dimension Error");
    const int64_t n = width;
    double* dA = A;
    int64_t ld = LineWidthA / 8;
    const bool direct = aligned16(A) && (LineWidthA & 15) == 0;
    if (!direct) {
        void* p;
        ld = padded_ld(n);
        B2M_TRY(ws_get(ctx, kWsMatA, (size_t)(n * ld * 8), &p));
        dA = (double*)p;
        B2M_TRY(copy_matrix(ctx, ctx->stream, dA, ld * 8, A, LineWidthA, n, n));
    }
    void* pp;
    B2M_TRY(ws_get(ctx, kWsPiv, (size_t)(2 * n * 4), &pp));
    B2M_CU(ctx, cudaMemsetAsync(indx, 0, (size_t)n * 4, ctx->stream));
    B2M_TRY(reset_status(ctx));
    B2M_TRY(lu_factor_f64(ctx, ctx->stream, dA, ld, n, indx, (int32_t*)pp + n));
    if (!direct) B2M_TRY(copy_matrix(ctx, ctx->stream, A, LineWidthA, dA, ld * 8, n, n));
    if (status) B2M_TRY(publish_status(ctx, ctx->stream, ctx->d_status, status));
    return B2M_OK;
}

extern "C" int32_t b2m_dev_MatrixLUBackSubst(b2m_ctx* h, const double* LUDecomp, int64_t LineWidthLU,
                                             int64_t width, const int32_t* indx, double* B, int64_t LineWidthB,
                                             int64_t nrhs) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!LUDecomp || !indx || !B) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (width <= 0 || nrhs <= 0 || !lw_ok(LineWidthLU, width) || !lw_ok(LineWidthB, nrhs))
        return fail(ctx, B2M_ERR_DIM, "Dimension Error");
    const int64_t n = width;
    const double* LU = LUDecomp;
    int64_t ld = LineWidthLU / 8;
    if (!aligned16(LU) || (LineWidthLU & 15)) {
        void* p;
        ld = padded_ld(n);
        B2M_TRY(ws_get(ctx, kWsMatA, (size_t)(n * ld * 8), &p));
        B2M_TRY(copy_matrix(ctx, ctx->stream, (double*)p, ld * 8, LUDecomp, LineWidthLU, n, n));
        LU = (const double*)p;
    }
    double* dB = B;
    int64_t ldb = LineWidthB / 8;
    const bool bdirect = aligned16(B) && (LineWidthB & 15) == 0;
    if (!bdirect) {
        void* p;
        ldb = padded_ld(nrhs);
        B2M_TRY(ws_get(ctx, kWsMatB, (size_t)(n * ldb * 8), &p));
        dB = (double*)p;
        B2M_TRY(copy_matrix(ctx, ctx->stream, dB, ldb * 8, B, LineWidthB, n, nrhs));
    }
    void* pp;
    B2M_TRY(ws_get(ctx, kWsPiv, (size_t)(2 * n * 4), &pp));
    int32_t* dperm = (int32_t*)pp + n;
    B2M_TRY(reset_status(ctx));
    B2M_TRY(perm_from_ipiv(ctx, ctx->stream, indx, n, dperm));
    B2M_TRY(lu_solve_f64(ctx, ctx->stream, LU, ld, n, dperm, dB, ldb, nrhs));
    if (!bdirect) B2M_TRY(copy_matrix(ctx, ctx->stream, B, LineWidthB, dB, ldb * 8, n, nrhs));
    return B2M_OK;
}

extern "C" int32_t b2m_dev_MatrixLinEQSolve(b2m_ctx* h, const double* A, int64_t LineWidthA, int64_t width,
                                            const double* B, int64_t LineWidthB, double* X, int64_t LineWidthX,
                                            int64_t Width2, int64_t NumRefinements, int32_t* status) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!A || !B || !X) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (width <= 0 || Width2 <= 0 || !lw_ok(LineWidthA, width) || !lw_ok(LineWidthB, Width2) ||
        !lw_ok(LineWidthX, Width2) || NumRefinements < 0)
        return fail(ctx, B2M_ERR_DIM, "Dimension error");
    const int64_t n = width, ld = padded_ld(n), ldb = padded_ld(Width2);
    void *pa, *pb, *px, *pp;
    B2M_TRY(ws_get(ctx, kWsMatA, (size_t)(n * ld * 8), &pa));
    B2M_TRY(ws_get(ctx, kWsMatB, (size_t)(n * ldb * 8), &pb));
    B2M_TRY(ws_get(ctx, kWsMatD, (size_t)(n * ldb * 8), &px));
    B2M_TRY(ws_get(ctx, kWsPiv, (size_t)(2 * n * 4), &pp));
    B2M_TRY(copy_matrix(ctx, ctx->stream, (double*)pa, ld * 8, A, LineWidthA, n, n));
    B2M_TRY(copy_matrix(ctx, ctx->stream, (double*)pb, ldb * 8, B, LineWidthB, n, Width2));
    const double* Ao = A;
    int64_t ldAo = LineWidthA / 8;
    if (NumRefinements > 0 && (!aligned16(A) || (LineWidthA & 15))) {
        void* pc;
        B2M_TRY(ws_get(ctx, kWsMatC, (size_t)(n * ld * 8), &pc));
        B2M_TRY(copy_matrix(ctx, ctx->stream, (double*)pc, ld * 8, A, LineWidthA, n, n));
        Ao = (const double*)pc;
        ldAo = ld;
    }
    B2M_TRY(reset_status(ctx));
    int32_t* dpiv = (int32_t*)pp;
    B2M_TRY(solve_device(ctx, (double*)pa, ld, n, Ao, ldAo, (double*)pb, ldb, (double*)px, ldb, Width2,
                         NumRefinements, dpiv, dpiv + n));
    B2M_TRY(copy_matrix(ctx, ctx->stream, X, LineWidthX, (double*)px, ldb * 8, n, Width2));
    if (status) B2M_TRY(publish_status(ctx, ctx->stream, ctx->d_status, status));
    return B2M_OK;
}

extern "C" int32_t b2m_dev_MatrixInverseInPlace(b2m_ctx* h, double* A, int64_t LineWidthA, int64_t width,
                                                int32_t* status) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!A) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (width <= 0 || !lw_ok(LineWidthA, width)) return fail(ctx, B2M_ERR_DIM, "Dimension Error");
    const int64_t n = width, ld = padded_ld(n);
    void *pa, *pb, *pp;
    B2M_TRY(ws_get(ctx, kWsMatA, (size_t)(n * ld * 8), &pa));
    B2M_TRY(ws_get(ctx, kWsMatB, (size_t)(n * ld * 8), &pb));
    B2M_TRY(ws_get(ctx, kWsPiv, (size_t)(2 * n * 4), &pp));
    double* dLU = (double*)pa;
    double* X = (double*)pb;
    int32_t* dpiv = (int32_t*)pp;
    B2M_TRY(copy_matrix(ctx, ctx->stream, dLU, ld * 8, A, LineWidthA, n, n));
    B2M_TRY(reset_status(ctx));
    B2M_TRY(lu_factor_f64(ctx, ctx->stream, dLU, ld, n, dpiv, dpiv + n));
    B2M_CU(ctx, cudaMemset2DAsync(X, ld * 8, 0, n * 8, n, ctx->stream));
    B2M_TRY(set_diagonal(ctx, ctx->stream, X, ld, n, 1.0));
    B2M_TRY(lu_solve_f64(ctx, ctx->stream, dLU, ld, n, dpiv + n, X, ld, n));
    // the inverse replaces A only when the factorisation succeeded
    B2M_TRY(copy_if_ok(ctx, ctx->stream, A, LineWidthA / 8, X, ld, n, n));
    if (status) B2M_TRY(publish_status(ctx, ctx->stream, ctx->d_status, status));
    return B2M_OK;
}

extern "C" int32_t b2m_dev_MatrixDeterminant(b2m_ctx* h, const double* A, int64_t LineWidthA, int64_t width,
                                             double* det) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!A || !det) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (width <= 0 || !lw_ok(LineWidthA, width)) return fail(ctx, B2M_ERR_DIM, "Dimension error");
    const int64_t n = width, ld = padded_ld(n);
    void *pa, *pp;
    B2M_TRY(ws_get(ctx, kWsMatA, (size_t)(n * ld * 8), &pa));
    B2M_TRY(ws_get(ctx, kWsPiv, (size_t)(2 * n * 4), &pp));
    B2M_TRY(copy_matrix(ctx, ctx->stream, (double*)pa, ld * 8, A, LineWidthA, n, n));
    B2M_TRY(reset_status(ctx));
    B2M_TRY(lu_factor_f64(ctx, ctx->stream, (double*)pa, ld, n, (int32_t*)pp, (int32_t*)pp + n));
    return lu_determinant(ctx, ctx->stream, (double*)pa, ld, n, (int32_t*)pp, det);
}

// ======================================================================================= mixed precision
namespace {
int32_t mixed_common(Ctx* ctx, const double* A, int64_t lda, int64_t n, const double* B, int64_t ldb, double* X,
                     int64_t ldx, int64_t nrhs, int32_t mode, int32_t maxIter, double tol, b2m_solve_report* report) {
    MixedReport rep{};
    const double t = tol > 0 ? tol : (double)n * std::ldexp(1.0, -53);
    const int defit = mode == B2M_MIXED_TF32 ? 30 : 10;  // TF32 contracts ~10x per step, 3xTF32 ~1e3x
    const int32_t st = solve_mixed(ctx, ctx->stream, A, lda, n, B, ldb, X, ldx, nrhs, mode,
                                   maxIter > 0 ? maxIter : defit, t, &rep);
    if (report) {
        report->iterations = rep.iterations;
        report->fell_back = rep.fell_back;
        report->backward_error = rep.backward_error;
        report->refinement_backward_error = rep.ir_backward_error;
        report->forward_error = rep.forward_error;
    }
    return st;
}
}  // namespace

extern "C" int32_t b2m_dev_MatrixLinEQSolveMixed(b2m_ctx* h, const double* A, int64_t LineWidthA, int64_t width,
                                                 const double* B, int64_t LineWidthB, double* X, int64_t LineWidthX,
                                                 int64_t Width2, int32_t mode, int32_t maxIter, double tol,
                                                 b2m_solve_report* report) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!A || !B || !X) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (width <= 0 || Width2 <= 0 || !lw_ok(LineWidthA, width) || !lw_ok(LineWidthB, Width2) ||
        !lw_ok(LineWidthX, Width2))
        return fail(ctx, B2M_ERR_DIM, "Dimension error");
    const int64_t n = width;
    const double* dA = A;
    int64_t lda = LineWidthA / 8;
    if (!aligned16(A) || (LineWidthA & 15)) {
        void* p;
        lda = padded_ld(n);
        B2M_TRY(ws_get(ctx, kWsMatA, (size_t)(n * lda * 8), &p));
        B2M_TRY(copy_matrix(ctx, ctx->stream, (double*)p, lda * 8, A, LineWidthA, n, n));
        dA = (const double*)p;
    }
    const double* dB = B;
    int64_t ldb = LineWidthB / 8;
    if (!aligned16(B) || (LineWidthB & 15)) {
        void* p;
        ldb = padded_ld(Width2);
        B2M_TRY(ws_get(ctx, kWsMatB, (size_t)(n * ldb * 8), &p));
        B2M_TRY(copy_matrix(ctx, ctx->stream, (double*)p, ldb * 8, B, LineWidthB, n, Width2));
        dB = (const double*)p;
    }
    double* dX = X;
    int64_t ldx = LineWidthX / 8;
    const bool xdirect = aligned16(X) && (LineWidthX & 15) == 0;
    if (!xdirect) {
        void* p;
        ldx = padded_ld(Width2);
        B2M_TRY(ws_get(ctx, kWsG, (size_t)(n * ldx * 8), &p));
        dX = (double*)p;
    }
    const int32_t st = mixed_common(ctx, dA, lda, n, dB, ldb, dX, ldx, Width2, mode, maxIter, tol, report);
    if (st == B2M_OK && !xdirect) B2M_TRY(copy_matrix(ctx, ctx->stream, X, LineWidthX, dX, ldx * 8, n, Width2));
    return st;
}

extern "C" int32_t b2m_MatrixLinEQSolveMixed(b2m_ctx* h, const double* A, int64_t LineWidthA, int64_t width,
                                             const double* B, int64_t LineWidthB, double* X, int64_t LineWidthX,
                                             int64_t Width2, int32_t mode, int32_t maxIter, double tol,
                                             b2m_solve_report* report) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!A || !B || !X) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (width <= 0 || Width2 <= 0 || !lw_ok(LineWidthA, width) || !lw_ok(LineWidthB, Width2) ||
        !lw_ok(LineWidthX, Width2))
        return fail(ctx, B2M_ERR_DIM, "Dimension error");
    cudaSetDevice(ctx->device);
    const int64_t n = width, lda = padded_ld(n), ldb = padded_ld(Width2);
    void *pa, *pb, *pxx;
    B2M_TRY(ws_get(ctx, kWsMatA, (size_t)(n * lda * 8), &pa));
    B2M_TRY(ws_get(ctx, kWsMatB, (size_t)(n * ldb * 8), &pb));
    B2M_TRY(ws_get(ctx, kWsG, (size_t)(n * ldb * 8), &pxx));
    B2M_TRY(upload(ctx, (double*)pa, lda, A, LineWidthA, n, n));
    B2M_TRY(upload(ctx, (double*)pb, ldb, B, LineWidthB, n, Width2));
    const int32_t st = mixed_common(ctx, (double*)pa, lda, n, (double*)pb, ldb, (double*)pxx, ldb, Width2, mode,
                                    maxIter, tol, report);
    if (st != B2M_OK) return st;
    B2M_TRY(download(ctx, X, LineWidthX, (double*)pxx, ldb, n, Width2));
    return finish(ctx);
}

// ------------------------------------------------------------------ adjoint solve (SolveLinEQAdjoint)
extern "C" int32_t b2m_dev_MatrixLinEQSolveAdjoint(b2m_ctx* h, const double* LUDecomp, int64_t LineWidthLU,
                                                   int64_t width, const int32_t* indx, const double* X,
                                                   int64_t LineWidthX, const double* G, int64_t LineWidthG,
                                                   int64_t nrhs, double* Lambda, int64_t LineWidthLambda, double* dA,
                                                   int64_t LineWidthdA, int32_t op) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!LUDecomp || !indx || !X || !G || !Lambda) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (op != B2M_DO_NONE && op != B2M_DO_ADD) return fail(ctx, B2M_ERR_ARG, "op must be B2M_DO_NONE or B2M_DO_ADD");
    const int64_t n = width;
    if (n <= 0 || nrhs <= 0 || !lw_ok(LineWidthLU, n) || !lw_ok(LineWidthX, nrhs) || !lw_ok(LineWidthG, nrhs) ||
        !lw_ok(LineWidthLambda, nrhs) || (dA && !lw_ok(LineWidthdA, n)))
        return fail(ctx, B2M_ERR_DIM, "Dimension Error");
    const int64_t ldy = padded_ld(nrhs);
    void *py, *pp;
    B2M_TRY(ws_get(ctx, kWsG, (size_t)(n * ldy * 8), &py));
    B2M_TRY(ws_get(ctx, kWsPiv, (size_t)(2 * n * 4), &pp));
    int32_t* dperm = (int32_t*)pp + n;
    B2M_TRY(reset_status(ctx));
    B2M_TRY(perm_from_ipiv(ctx, ctx->stream, indx, n, dperm));
    B2M_TRY(solve_adjoint_f64(ctx, ctx->stream, LUDecomp, LineWidthLU / 8, n, dperm, X, LineWidthX / 8, G,
                              LineWidthG / 8, nrhs, Lambda, LineWidthLambda / 8, dA, LineWidthdA / 8, op, (double*)py,
                              ldy));
    return B2M_OK;
}

extern "C" int32_t b2m_MatrixLinEQSolveAdjoint(b2m_ctx* h, const double* LUDecomp, int64_t LineWidthLU, int64_t width,
                                               const int32_t* indx, const double* X, int64_t LineWidthX,
                                               const double* G, int64_t LineWidthG, int64_t nrhs, double* Lambda,
                                               int64_t LineWidthLambda, double* dA, int64_t LineWidthdA, int32_t op) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!LUDecomp || !indx || !X || !G || !Lambda) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (op != B2M_DO_NONE && op != B2M_DO_ADD) return fail(ctx, B2M_ERR_ARG, "op must be B2M_DO_NONE or B2M_DO_ADD");
    const int64_t n = width;
    if (n <= 0 || nrhs <= 0 || !lw_ok(LineWidthLU, n) || !lw_ok(LineWidthX, nrhs) || !lw_ok(LineWidthG, nrhs) ||
        !lw_ok(LineWidthLambda, nrhs) || (dA && !lw_ok(LineWidthdA, n)))
        return fail(ctx, B2M_ERR_DIM, "Dimension Error");
    cudaSetDevice(ctx->device);
    const int64_t ld = padded_ld(n), ldk = padded_ld(nrhs);
    void *pa, *px, *pg, *py, *pl, *pd = nullptr, *pp;
    B2M_TRY(ws_get(ctx, kWsMatA, (size_t)(n * ld * 8), &pa));
    B2M_TRY(ws_get(ctx, kWsMatB, (size_t)(n * ldk * 8), &px));
    B2M_TRY(ws_get(ctx, kWsE, (size_t)(n * ldk * 8), &pg));
    B2M_TRY(ws_get(ctx, kWsF, (size_t)(n * ldk * 8), &pl));
    B2M_TRY(ws_get(ctx, kWsG, (size_t)(n * ldk * 8), &py));
    if (dA) B2M_TRY(ws_get(ctx, kWsMatC, (size_t)(n * ld * 8), &pd));
    B2M_TRY(ws_get(ctx, kWsPiv, (size_t)(2 * n * 4), &pp));
    int32_t* dpiv = (int32_t*)pp;
    int32_t* dperm = dpiv + n;
    B2M_TRY(upload(ctx, (double*)pa, ld, LUDecomp, LineWidthLU, n, n));
    B2M_TRY(upload(ctx, (double*)px, ldk, X, LineWidthX, n, nrhs));
    B2M_TRY(upload(ctx, (double*)pg, ldk, G, LineWidthG, n, nrhs));
    if (dA && op == B2M_DO_ADD) B2M_TRY(upload(ctx, (double*)pd, ld, dA, LineWidthdA, n, n));
    B2M_CU(ctx, cudaMemcpyAsync(dpiv, indx, (size_t)n * 4, cudaMemcpyHostToDevice, ctx->stream));
    B2M_TRY(reset_status(ctx));
    B2M_TRY(perm_from_ipiv(ctx, ctx->stream, dpiv, n, dperm));
    B2M_TRY(solve_adjoint_f64(ctx, ctx->stream, (double*)pa, ld, n, dperm, (double*)px, ldk, (double*)pg, ldk, nrhs,
                              (double*)pl, ldk, (double*)pd, ld, op, (double*)py, ldk));
    B2M_TRY(download(ctx, Lambda, LineWidthLambda, (double*)pl, ldk, n, nrhs));
    if (dA) B2M_TRY(download(ctx, dA, LineWidthdA, (double*)pd, ld, n, n));
    return finish(ctx);
}

// ------------------------------------------------------------------ batched uneven solves
namespace {
int32_t batch_check(Ctx* ctx, int64_t count, const int32_t* n, const int32_t* nrhs, const int64_t* a_off,
                    const int64_t* b_off, int64_t* a_elems, int64_t* b_elems) {
    if (count < 0) return fail(ctx, B2M_ERR_DIM, "count < 0");
    if (count > 0 && (!n || !nrhs || !a_off || !b_off)) return fail(ctx, B2M_ERR_ARG, "null plan array");
    int64_t ae = 0, be = 0;
    for (int64_t i = 0; i < count; ++i) {
        if (a_off[i] < 0 || b_off[i] < 0) return fail(ctx, B2M_ERR_DIM, "negative offset");
        ae = std::max(ae, a_off[i] + (int64_t)n[i] * n[i]);
        be = std::max(be, b_off[i] + (int64_t)n[i] * nrhs[i]);
    }
    *a_elems = ae;
    *b_elems = be;
    return B2M_OK;
}
}  // namespace

extern "C" int32_t b2m_dev_BatchLinEQSolve(b2m_ctx* h, int64_t count, const int32_t* n, const int32_t* nrhs,
                                           const int64_t* a_off, const int64_t* b_off, const double* A,
                                           const double* B, double* X, int32_t mode, int32_t* info, int32_t* iters) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    int64_t ae, be;
    B2M_TRY(batch_check(ctx, count, n, nrhs, a_off, b_off, &ae, &be));
    if (count == 0) return B2M_OK;
    if (!A || !B || !X || !info) return fail(ctx, B2M_ERR_ARG, "null pointer");
    return batch_solve(ctx, ctx->stream, count, n, nrhs, a_off, b_off, A, B, X, mode, info, iters, nullptr);
}

extern "C" int32_t b2m_BatchLinEQSolve(b2m_ctx* h, int64_t count, const int32_t* n, const int32_t* nrhs,
                                       const int64_t* a_off, const int64_t* b_off, const double* A, const double* B,
                                       double* X, int32_t mode, int32_t* info, int32_t* iters) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    int64_t ae, be;
    B2M_TRY(batch_check(ctx, count, n, nrhs, a_off, b_off, &ae, &be));
    if (count == 0) return B2M_OK;
    if (!A || !B || !X || !info) return fail(ctx, B2M_ERR_ARG, "null pointer");
    cudaSetDevice(ctx->device);
    void *pa, *pb, *px, *pi;
    B2M_TRY(ws_get(ctx, kWsMatA, (size_t)ae * 8, &pa));
    B2M_TRY(ws_get(ctx, kWsMatB, (size_t)be * 8, &pb));
    B2M_TRY(ws_get(ctx, kWsMatC, (size_t)be * 8, &px));
    B2M_TRY(ws_get(ctx, kWsE, (size_t)count * 8, &pi));
    int32_t* dinfo = (int32_t*)pi;
    int32_t* diters = dinfo + count;
    B2M_CU(ctx, cudaMemcpyAsync(pa, A, (size_t)ae * 8, cudaMemcpyHostToDevice, ctx->stream));
    B2M_CU(ctx, cudaMemcpyAsync(pb, B, (size_t)be * 8, cudaMemcpyHostToDevice, ctx->stream));
    B2M_TRY(reset_status(ctx));
    B2M_TRY(batch_solve(ctx, ctx->stream, count, n, nrhs, a_off, b_off, (const double*)pa, (const double*)pb,
                        (double*)px, mode, dinfo, diters, nullptr));
    B2M_CU(ctx, cudaMemcpyAsync(X, px, (size_t)be * 8, cudaMemcpyDeviceToHost, ctx->stream));
    B2M_CU(ctx, cudaMemcpyAsync(info, dinfo, (size_t)count * 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (iters) B2M_CU(ctx, cudaMemcpyAsync(iters, diters, (size_t)count * 4, cudaMemcpyDeviceToHost, ctx->stream));
    B2M_CU(ctx, cudaStreamSynchronize(ctx->stream));
    return B2M_OK;
}

extern "C" int32_t b2m_batch_tune_read(b2m_ctx* h, int32_t* small_n, int32_t* group_warps, int32_t* pw_large,
                                       int32_t* pw_small, float* ms) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (ctx->batch_tunes.empty()) return fail(ctx, B2M_ERR_ARG, "no batch has been tuned yet");
    const BatchTune& t = ctx->batch_tunes.find(ctx->batch_plan_sig) != ctx->batch_tunes.end()
                             ? ctx->batch_tunes[ctx->batch_plan_sig]
                             : ctx->batch_tunes.begin()->second;
    if (small_n) *small_n = t.small_n;
    if (group_warps) *group_warps = t.group_warps;
    if (pw_large) *pw_large = t.pw_large;
    if (pw_small) *pw_small = t.pw_small;
    if (ms) *ms = t.ms;
    return B2M_OK;
}

// ------------------------------------------------------------------ Ozaki split-precision GEMM
extern "C" int32_t b2m_dev_MatrixMultOzaki(b2m_ctx* h, double* dest, int64_t destLineWidth, const double* mt1,
                                           const double* mt2, int64_t width1, int64_t height1, int64_t width2,
                                           int64_t height2, int64_t LineWidth1, int64_t LineWidth2, int32_t op,
                                           int32_t slices) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!dest || !mt1 || !mt2) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (op < 0 || op > 2) return fail(ctx, B2M_ERR_ARG, "invalid op");
    if (width1 != height2 || width1 < 0 || height1 < 0 || width2 < 0)
        return fail(ctx, B2M_ERR_DIM, "Dimension error");
    if (!lw_ok(LineWidth1, width1) || !lw_ok(LineWidth2, width2) || !lw_ok(destLineWidth, width2))
        return fail(ctx, B2M_ERR_DIM, "Line widths do not match");
    return ozaki_gemm(ctx, ctx->stream, mt1, LineWidth1 / 8, mt2, LineWidth2 / 8, dest, destLineWidth / 8, height1,
                      width2, width1, op, slices <= 0 ? 8 : slices);
}

extern "C" int32_t b2m_MatrixMultOzaki(b2m_ctx* h, double* dest, int64_t destLineWidth, const double* mt1,
                                       const double* mt2, int64_t width1, int64_t height1, int64_t width2,
                                       int64_t height2, int64_t LineWidth1, int64_t LineWidth2, int32_t op,
                                       int32_t slices) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!dest || !mt1 || !mt2) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (op < 0 || op > 2) return fail(ctx, B2M_ERR_ARG, "invalid op");
    if (width1 != height2 || width1 < 0 || height1 < 0 || width2 < 0)
        return fail(ctx, B2M_ERR_DIM, "Dimension error");
    if (!lw_ok(LineWidth1, width1) || !lw_ok(LineWidth2, width2) || !lw_ok(destLineWidth, width2))
        return fail(ctx, B2M_ERR_DIM, "Line widths do not match");
    if (height1 == 0 || width2 == 0) return B2M_OK;
    cudaSetDevice(ctx->device);
    const int64_t M = height1, N = width2, K = width1;
    const int64_t lda = padded_ld(K), ldb = padded_ld(N);
    void *pa, *pb, *pc;
    B2M_TRY(ws_get(ctx, kWsMatA, (size_t)(std::max<int64_t>(M, 1) * lda * 8), &pa));
    B2M_TRY(ws_get(ctx, kWsMatB, (size_t)(std::max<int64_t>(K, 1) * ldb * 8), &pb));
    B2M_TRY(ws_get(ctx, kWsMatC, (size_t)(M * ldb * 8), &pc));
    if (K > 0) {
        B2M_TRY(upload(ctx, (double*)pa, lda, mt1, LineWidth1, M, K));
        B2M_TRY(upload(ctx, (double*)pb, ldb, mt2, LineWidth2, K, N));
    }
    if (op != B2M_DO_NONE) B2M_TRY(upload(ctx, (double*)pc, ldb, dest, destLineWidth, M, N));
    B2M_TRY(reset_status(ctx));
    B2M_TRY(ozaki_gemm(ctx, ctx->stream, (double*)pa, lda, (double*)pb, ldb, (double*)pc, ldb, M, N, K, op,
                       slices <= 0 ? 8 : slices));
    B2M_TRY(download(ctx, dest, destLineWidth, (double*)pc, ldb, M, N));
    return finish(ctx);
}

// ======================================================================================= GEMM error report
namespace {

int32_t fill_gemm_report(Ctx* ctx, int32_t trans, const MultShape& s, const double* C, int64_t ldc, const double* A,
                         int64_t lda, const double* B, int64_t ldb, int32_t rows, b2m_gemm_report* rep) {
    double acc[4];
    const int nrows = (int)std::min<int64_t>(rows <= 0 ? 16 : rows, s.M);
    B2M_TRY(gemm_error_report(ctx, ctx->stream, C, ldc, A, lda, trans != 1, B, ldb, trans != 2, s.M, s.N, s.K, nrows,
                              acc));
    rep->rows_checked = nrows;
    rep->reserved = 0;
    rep->forward_error = acc[1] > 0 ? acc[0] / acc[1] : acc[0];
    rep->relative_error = acc[3] > 0 ? std::sqrt(acc[2] / acc[3]) : std::sqrt(acc[2]);
    rep->bound = (double)s.K * std::ldexp(1.0, -53);
    return B2M_OK;
}

}  // namespace

extern "C" int32_t b2m_dev_MatrixMultErrorReport(b2m_ctx* h, const double* dest, int64_t destLineWidth,
                                                 const double* mt1, const double* mt2, int64_t width1,
                                                 int64_t height1, int64_t width2, int64_t height2, int64_t LineWidth1,
                                                 int64_t LineWidth2, int32_t trans, int32_t sample_rows,
                                                 b2m_gemm_report* report) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!dest || !mt1 || !mt2 || !report) return fail(ctx, B2M_ERR_ARG, "null pointer");
    MultShape s;
    B2M_TRY(mult_shape(ctx, trans, width1, height1, width2, height2, &s));
    if (!lw_ok(LineWidth1, width1) || !lw_ok(LineWidth2, width2) || !lw_ok(destLineWidth, s.N))
        return fail(ctx, B2M_ERR_DIM, "Line widths do not match");
    *report = b2m_gemm_report{};
    if (s.M == 0 || s.N == 0) return B2M_OK;
    cudaSetDevice(ctx->device);
    return fill_gemm_report(ctx, trans, s, dest, destLineWidth / 8, mt1, LineWidth1 / 8, mt2, LineWidth2 / 8,
                            sample_rows, report);
}

extern "C" int32_t b2m_MatrixMultErrorReport(b2m_ctx* h, const double* dest, int64_t destLineWidth, const double* mt1,
                                             const double* mt2, int64_t width1, int64_t height1, int64_t width2,
                                             int64_t height2, int64_t LineWidth1, int64_t LineWidth2, int32_t trans,
                                             int32_t sample_rows, b2m_gemm_report* report) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!dest || !mt1 || !mt2 || !report) return fail(ctx, B2M_ERR_ARG, "null pointer");
    MultShape s;
    B2M_TRY(mult_shape(ctx, trans, width1, height1, width2, height2, &s));
    if (!lw_ok(LineWidth1, width1) || !lw_ok(LineWidth2, width2) || !lw_ok(destLineWidth, s.N))
        return fail(ctx, B2M_ERR_DIM, "Line widths do not match");
    *report = b2m_gemm_report{};
    if (s.M == 0 || s.N == 0) return B2M_OK;
    cudaSetDevice(ctx->device);
    const int64_t lda = padded_ld(width1), ldb = padded_ld(width2), ldc = padded_ld(s.N);
    void *pa, *pb, *pc;
    B2M_TRY(ws_get(ctx, kWsMatA, (size_t)(std::max<int64_t>(height1, 1) * lda * 8), &pa));
    B2M_TRY(ws_get(ctx, kWsMatB, (size_t)(std::max<int64_t>(height2, 1) * ldb * 8), &pb));
    B2M_TRY(ws_get(ctx, kWsMatC, (size_t)(s.M * ldc * 8), &pc));
    B2M_TRY(upload(ctx, (double*)pa, lda, mt1, LineWidth1, height1, width1));
    B2M_TRY(upload(ctx, (double*)pb, ldb, mt2, LineWidth2, height2, width2));
    B2M_TRY(upload(ctx, (double*)pc, ldc, dest, destLineWidth, s.M, s.N));
    return fill_gemm_report(ctx, trans, s, (double*)pc, ldc, (double*)pa, lda, (double*)pb, ldb, sample_rows, report);
}

// ======================================================================================= Cholesky
extern "C" int32_t b2m_MatrixCholeskyInPlace4(b2m_ctx* h, double* A, int64_t LineWidthA, int64_t width,
                                              int64_t pnlSize) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!A) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (width <= 0 || !lw_ok(LineWidthA, width) || pnlSize < 0) return fail(ctx, B2M_ERR_DIM, "Dimension error");
    cudaSetDevice(ctx->device);
    const int64_t ld = padded_ld(width);
    void *po, *pf;
    B2M_TRY(ws_get(ctx, kWsMatA, (size_t)(width * ld * 8), &po));
    B2M_TRY(ws_get(ctx, kWsMatC, (size_t)(width * ld * 8), &pf));
    double *orig = (double*)po, *F = (double*)pf;
    B2M_TRY(upload(ctx, orig, ld, A, LineWidthA, width, width));
    B2M_TRY(reset_status(ctx));
    B2M_TRY(copy_matrix(ctx, ctx->stream, F, ld * 8, orig, ld * 8, width, width));
    B2M_TRY(chol_factor_f64(ctx, ctx->stream, F, ld, width));
    // the caller's strict upper triangle comes back unchanged, as MatrixCholeskyInPlace4 leaves it
    B2M_TRY(copy_lower(ctx, ctx->stream, orig, ld, F, ld, width, true));
    B2M_TRY(download(ctx, A, LineWidthA, orig, ld, width, width));
    return finish(ctx);
}

extern "C" int32_t b2m_dev_MatrixCholeskyInPlace4(b2m_ctx* h, double* A, int64_t LineWidthA, int64_t width,
                                                  int32_t* status) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!A) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (width <= 0 || !lw_ok(LineWidthA, width)) return fail(ctx, B2M_ERR_DIM, "Dimension error");
    const int64_t ld = padded_ld(width);
    void* pf;
    B2M_TRY(ws_get(ctx, kWsMatC, (size_t)(width * ld * 8), &pf));
    double* F = (double*)pf;
    B2M_TRY(reset_status(ctx));
    B2M_TRY(copy_matrix(ctx, ctx->stream, F, ld * 8, A, LineWidthA, width, width));
    B2M_TRY(chol_factor_f64(ctx, ctx->stream, F, ld, width));
    B2M_TRY(copy_lower(ctx, ctx->stream, A, LineWidthA / 8, F, ld, width, true));
    if (status) B2M_TRY(publish_status(ctx, ctx->stream, ctx->d_status, status));
    return B2M_OK;
}

extern "C" int32_t b2m_MatrixCholeskyInPlace(b2m_ctx* h, double* A, int64_t LineWidthA, int64_t width, double* P,
                                             int64_t LineWidthP) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!A || !P) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (width <= 0 || !lw_ok(LineWidthA, width) || LineWidthP < 8 || (LineWidthP % 8))
        return fail(ctx, B2M_ERR_DIM, "Dimension error");
    cudaSetDevice(ctx->device);
    const int64_t ld = padded_ld(width), ldp = LineWidthP / 8;
    void *po, *pf, *pp;
    B2M_TRY(ws_get(ctx, kWsMatA, (size_t)(width * ld * 8), &po));
    B2M_TRY(ws_get(ctx, kWsMatC, (size_t)(width * ld * 8), &pf));
    B2M_TRY(ws_get(ctx, kWsF, (size_t)(width * ldp * 8), &pp));
    double *orig = (double*)po, *F = (double*)pf, *dP = (double*)pp;
    B2M_TRY(upload(ctx, orig, ld, A, LineWidthA, width, width));
    B2M_TRY(upload(ctx, dP, ldp, P, LineWidthP, width, 1));
    B2M_TRY(reset_status(ctx));
    B2M_TRY(copy_matrix(ctx, ctx->stream, F, ld * 8, orig, ld * 8, width, width));
    B2M_TRY(chol_factor_f64(ctx, ctx->stream, F, ld, width));
    // MatrixCholeskyInPlace (LinAlgCholesky.pas:270-332): L below the diagonal, the diagonal in P;
    // A's diagonal and upper triangle stay as they were
    B2M_TRY(split_nr(ctx, ctx->stream, orig, ld, dP, LineWidthP, F, ld, width));
    B2M_TRY(download(ctx, A, LineWidthA, orig, ld, width, width));
    B2M_TRY(download(ctx, P, LineWidthP, dP, ldp, width, 1));
    return finish(ctx);
}

namespace {
// A X = B with the factor in F (lower with diagonal), or in Lnr + P (NR form) when P is not null
int32_t chol_solve_dev(Ctx* ctx, const double* A, int64_t ldA, int64_t width, const double* P, int64_t LineWidthP,
                       double* X, int64_t ldx, int64_t nrhs) {
    const int64_t ld = padded_ld(width);
    void* pw;
    B2M_TRY(ws_get(ctx, kWsMatC, (size_t)(width * ld * 8), &pw));
    double* W = (double*)pw;
    if (P) {
        void* pf;
        B2M_TRY(ws_get(ctx, kWsMatD, (size_t)(width * ld * 8), &pf));
        B2M_TRY(join_nr(ctx, ctx->stream, (double*)pf, ld, A, ldA, P, LineWidthP, width));
        return chol_solve_f64(ctx, ctx->stream, (double*)pf, ld, width, W, ld, X, ldx, nrhs);
    }
    return chol_solve_f64(ctx, ctx->stream, A, ldA, width, W, ld, X, ldx, nrhs);
}
}  // namespace

extern "C" int32_t b2m_MatrixCholeskySolveLinEq(b2m_ctx* h, const double* A, int64_t LineWidthA, int64_t width,
                                                const double* P, int64_t LineWidthP, const double* B,
                                                int64_t LineWidthB, double* X, int64_t LineWidthX, int64_t nrhs) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!A || !B || !X) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (width <= 0 || nrhs <= 0 || !lw_ok(LineWidthA, width) || !lw_ok(LineWidthB, nrhs) || !lw_ok(LineWidthX, nrhs) ||
        (P && (LineWidthP < 8 || (LineWidthP % 8))))
        return fail(ctx, B2M_ERR_DIM, "Dimension error");
    cudaSetDevice(ctx->device);
    const int64_t ld = padded_ld(width), ldx = padded_ld(nrhs), ldp = P ? LineWidthP / 8 : 1;
    void *pa, *px, *pp = nullptr;
    B2M_TRY(ws_get(ctx, kWsMatA, (size_t)(width * ld * 8), &pa));
    B2M_TRY(ws_get(ctx, kWsMatB, (size_t)(width * ldx * 8), &px));
    if (P) B2M_TRY(ws_get(ctx, kWsF, (size_t)(width * ldp * 8), &pp));
    B2M_TRY(upload(ctx, (double*)pa, ld, A, LineWidthA, width, width));
    B2M_TRY(upload(ctx, (double*)px, ldx, B, LineWidthB, width, nrhs));
    if (P) B2M_TRY(upload(ctx, (double*)pp, ldp, P, LineWidthP, width, 1));
    B2M_TRY(reset_status(ctx));
    B2M_TRY(chol_solve_dev(ctx, (double*)pa, ld, width, (double*)pp, LineWidthP, (double*)px, ldx, nrhs));
    B2M_TRY(download(ctx, X, LineWidthX, (double*)px, ldx, width, nrhs));
    return finish(ctx);
}

extern "C" int32_t b2m_dev_MatrixCholeskySolveLinEq(b2m_ctx* h, const double* A, int64_t LineWidthA, int64_t width,
                                                    const double* P, int64_t LineWidthP, const double* B,
                                                    int64_t LineWidthB, double* X, int64_t LineWidthX, int64_t nrhs) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!A || !B || !X) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (width <= 0 || nrhs <= 0 || !lw_ok(LineWidthA, width) || !lw_ok(LineWidthB, nrhs) || !lw_ok(LineWidthX, nrhs) ||
        (P && (LineWidthP < 8 || (LineWidthP % 8))))
        return fail(ctx, B2M_ERR_DIM, "Dimension error");
    // the sweeps need an even, 16-byte aligned X; a caller X that is not gets a padded copy
    double* Xd = X;
    int64_t ldx = LineWidthX / 8;
    if (!aligned16(X) || (ldx & 1)) {
        void* p;
        ldx = padded_ld(nrhs);
        B2M_TRY(ws_get(ctx, kWsG, (size_t)(width * ldx * 8), &p));
        Xd = (double*)p;
    }
    B2M_TRY(copy_matrix(ctx, ctx->stream, Xd, ldx * 8, B, LineWidthB, width, nrhs));
    B2M_TRY(chol_solve_dev(ctx, A, LineWidthA / 8, width, P, LineWidthP, Xd, ldx, nrhs));
    if (Xd != X) B2M_TRY(copy_matrix(ctx, ctx->stream, X, LineWidthX, Xd, ldx * 8, width, nrhs));
    return B2M_OK;
}

// ======================================================================================= complex LU
namespace {

// a TComplex matrix (16 bytes per element, byte stride) on the device as two planes
struct ZPlanes {
    double *re, *im;
    int64_t ld;
};

bool zlw_ok(int64_t lw, int64_t cols) { return lw >= cols * 16 && (lw % 16) == 0; }

// host TComplex rows x cols -> planes in `slot` (the interleaved staging copy goes to kWsF)
int32_t z_upload(Ctx* ctx, int slot, const double* host, int64_t lw, int64_t rows, int64_t cols, ZPlanes* out) {
    const int64_t ld = padded_ld(cols);
    void *pp, *ps;
    B2M_TRY(ws_get(ctx, slot, (size_t)(2 * std::max<int64_t>(rows, 1) * ld * 8), &pp));
    const int64_t lds = round_up(cols * 16, 128);
    B2M_TRY(ws_get(ctx, kWsF, (size_t)(std::max<int64_t>(rows, 1) * lds), &ps));
    *out = ZPlanes{(double*)pp, (double*)pp + rows * ld, ld};
    B2M_CU(ctx, cudaMemcpy2DAsync(ps, lds, host, lw, cols * 16, rows, cudaMemcpyHostToDevice, ctx->stream));
    return z_deinterleave(ctx, ctx->stream, (const double*)ps, lds, out->re, out->im, ld, rows, cols);
}

int32_t z_download(Ctx* ctx, const ZPlanes& p, double* host, int64_t lw, int64_t rows, int64_t cols, bool only_if_ok) {
    const int64_t lds = round_up(cols * 16, 128);
    void* ps;
    B2M_TRY(ws_get(ctx, kWsF, (size_t)(std::max<int64_t>(rows, 1) * lds), &ps));
    if (only_if_ok)  // keep the caller's data when the factorisation stopped: stage it first
        B2M_CU(ctx, cudaMemcpy2DAsync(ps, lds, host, lw, cols * 16, rows, cudaMemcpyHostToDevice, ctx->stream));
    B2M_TRY(z_interleave(ctx, ctx->stream, (double*)ps, lds, p.re, p.im, p.ld, rows, cols, only_if_ok));
    B2M_CU(ctx, cudaMemcpy2DAsync(host, lw, ps, lds, cols * 16, rows, cudaMemcpyDeviceToHost, ctx->stream));
    return B2M_OK;
}

int32_t z_factor_host(Ctx* ctx, const double* A, int64_t lwA, int64_t n, ZPlanes* P, int32_t** dpiv, int32_t** dperm) {
    B2M_TRY(z_upload(ctx, kWsMatA, A, lwA, n, n, P));
    void* pp;
    B2M_TRY(ws_get(ctx, kWsPiv, (size_t)(2 * n * 4), &pp));
    *dpiv = (int32_t*)pp;
    *dperm = *dpiv + n;
    B2M_CU(ctx, cudaMemsetAsync(*dpiv, 0, (size_t)n * 4, ctx->stream));
    B2M_TRY(reset_status(ctx));
    return zlu_factor(ctx, ctx->stream, P->re, P->im, P->ld, n, *dpiv, *dperm);
}

}  // namespace

extern "C" int32_t b2m_CplxMatrixLUDecompInPlace(b2m_ctx* h, double* A, int64_t LineWidthA, int64_t width,
                                                 int32_t* indx) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!A || !indx) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (width <= 0 || !zlw_ok(LineWidthA, width)) return fail(ctx, B2M_ERR_DIM, "Dimension Error");
    cudaSetDevice(ctx->device);
    std::memset(indx, 0, (size_t)width * sizeof(int32_t));
    ZPlanes P;
    int32_t *dpiv, *dperm;
    B2M_TRY(z_factor_host(ctx, A, LineWidthA, width, &P, &dpiv, &dperm));
    B2M_TRY(z_download(ctx, P, A, LineWidthA, width, width, false));
    B2M_CU(ctx, cudaMemcpyAsync(indx, dpiv, (size_t)width * 4, cudaMemcpyDeviceToHost, ctx->stream));
    return finish(ctx);
}

extern "C" int32_t b2m_CplxMatrixLUBackSubst(b2m_ctx* h, const double* LUDecomp, int64_t LineWidthLU, int64_t width,
                                             const int32_t* indx, double* B, int64_t LineWidthB, int64_t nrhs) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!LUDecomp || !indx || !B) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (width <= 0 || nrhs <= 0 || !zlw_ok(LineWidthLU, width) || !zlw_ok(LineWidthB, nrhs))
        return fail(ctx, B2M_ERR_DIM, "Dimension Error");
    cudaSetDevice(ctx->device);
    ZPlanes L, X;
    B2M_TRY(z_upload(ctx, kWsMatA, LUDecomp, LineWidthLU, width, width, &L));
    B2M_TRY(z_upload(ctx, kWsMatB, B, LineWidthB, width, nrhs, &X));
    void *pp, *pt;
    B2M_TRY(ws_get(ctx, kWsPiv, (size_t)(2 * width * 4), &pp));
    B2M_TRY(ws_get(ctx, kWsE, (size_t)(2 * width * X.ld * 8), &pt));
    int32_t* dpiv = (int32_t*)pp;
    B2M_CU(ctx, cudaMemcpyAsync(dpiv, indx, (size_t)width * 4, cudaMemcpyHostToDevice, ctx->stream));
    B2M_TRY(reset_status(ctx));
    B2M_TRY(perm_from_ipiv(ctx, ctx->stream, dpiv, width, dpiv + width));
    B2M_TRY(zlu_solve(ctx, ctx->stream, L.re, L.im, L.ld, width, dpiv + width, X.re, X.im, X.ld, nrhs, (double*)pt,
                      (double*)pt + width * X.ld));
    B2M_TRY(z_download(ctx, X, B, LineWidthB, width, nrhs, false));
    return finish(ctx);
}

extern "C" int32_t b2m_CplxMatrixLinEQSolve(b2m_ctx* h, const double* A, int64_t LineWidthA, int64_t width,
                                            const double* B, int64_t LineWidthB, double* X, int64_t LineWidthX,
                                            int64_t Width2) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!A || !B || !X) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (width <= 0 || Width2 <= 0 || !zlw_ok(LineWidthA, width) || !zlw_ok(LineWidthB, Width2) ||
        !zlw_ok(LineWidthX, Width2))
        return fail(ctx, B2M_ERR_DIM, "Dimension Error");
    cudaSetDevice(ctx->device);
    ZPlanes P, Xp;
    int32_t *dpiv, *dperm;
    B2M_TRY(z_factor_host(ctx, A, LineWidthA, width, &P, &dpiv, &dperm));
    B2M_TRY(z_upload(ctx, kWsMatB, B, LineWidthB, width, Width2, &Xp));
    void* pt;
    B2M_TRY(ws_get(ctx, kWsE, (size_t)(2 * width * Xp.ld * 8), &pt));
    B2M_TRY(zlu_solve(ctx, ctx->stream, P.re, P.im, P.ld, width, dperm, Xp.re, Xp.im, Xp.ld, Width2, (double*)pt,
                      (double*)pt + width * Xp.ld));
    B2M_TRY(z_download(ctx, Xp, X, LineWidthX, width, Width2, false));
    return finish(ctx);
}

extern "C" int32_t b2m_CplxMatrixInverseInPlace(b2m_ctx* h, double* A, int64_t LineWidthA, int64_t width) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!A) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (width <= 0 || !zlw_ok(LineWidthA, width)) return fail(ctx, B2M_ERR_DIM, "Dimension Error");
    cudaSetDevice(ctx->device);
    ZPlanes P;
    int32_t *dpiv, *dperm;
    B2M_TRY(z_factor_host(ctx, A, LineWidthA, width, &P, &dpiv, &dperm));
    // the columns of the inverse: solves with the identity (CplxMatrixInverseInPlace :1531-1548)
    const int64_t ld = padded_ld(width);
    void *pi, *pt;
    B2M_TRY(ws_get(ctx, kWsMatB, (size_t)(2 * width * ld * 8), &pi));
    B2M_TRY(ws_get(ctx, kWsE, (size_t)(2 * width * ld * 8), &pt));
    ZPlanes I{(double*)pi, (double*)pi + width * ld, ld};
    B2M_CU(ctx, cudaMemsetAsync(pi, 0, (size_t)(2 * width * ld * 8), ctx->stream));
    B2M_TRY(set_diagonal(ctx, ctx->stream, I.re, ld, width, 1.0));
    B2M_TRY(zlu_solve(ctx, ctx->stream, P.re, P.im, P.ld, width, dperm, I.re, I.im, ld, width, (double*)pt,
                      (double*)pt + width * ld));
    B2M_TRY(z_download(ctx, I, A, LineWidthA, width, width, true));  // A is left as it was when singular
    return finish(ctx);
}

extern "C" int32_t b2m_CplxMatrixDeterminant(b2m_ctx* h, const double* A, int64_t LineWidthA, int64_t width,
                                             double* det) {
    Ctx* ctx = as_ctx(h);
    if (!ctx) return B2M_ERR_ARG;
    CallLock lk(ctx);
    if (!A || !det) return fail(ctx, B2M_ERR_ARG, "null pointer");
    if (width <= 0 || !zlw_ok(LineWidthA, width)) return fail(ctx, B2M_ERR_DIM, "Dimension error");
    cudaSetDevice(ctx->device);
    ZPlanes P;
    int32_t *dpiv, *dperm;
    B2M_TRY(z_factor_host(ctx, A, LineWidthA, width, &P, &dpiv, &dperm));
    void* pd;
    B2M_TRY(ws_get(ctx, kWsSmall, 2 * sizeof(double), &pd));
    B2M_TRY(z_determinant(ctx, ctx->stream, P.re, P.im, P.ld, width, dpiv, (double*)pd));
    B2M_CU(ctx, cudaMemcpyAsync(det, pd, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    const int32_t r = finish(ctx);
    return r == B2M_SINGULAR ? B2M_OK : r;  // a singular matrix has determinant 0, status leOk (:1578-1584)
}
