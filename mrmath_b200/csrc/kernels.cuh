// kernels.cuh -- internal launch interfaces shared by the translation units of libb2m.
#pragma once

#include "common.cuh"

namespace b2m {

// One GEMM operand as seen by the TMA tensor map: the map covers `rows x cols` elements of a
// row-major array at `base` with row stride `ld` (elements); the operand starts at (r0, c0)
// inside it.  kmajor: rows index m (A) or n (B) and cols index k; otherwise rows index k.
struct DOperand {
    const void* base;
    int64_t ld;
    int64_t rows, cols;
    int64_t r0, c0;
    bool kmajor;
};

// C(M x N) op= A(M x K) * B(K x N) in FP64 on the DMMA path.  Tensor-map origins c0 must be
// even; any K works (a k range that ends inside the maps off the 16-wide k-tile runs its last
// K % 16 columns as a separate short-K pass).
int32_t dgemm_tiled(Ctx* ctx, cudaStream_t st, const DOperand& A, const DOperand& B, double* C, int64_t ldc,
                    int64_t M, int64_t N, int64_t K, int op, bool check_info);

// Partial-pivoting LU of the leading n x n block of a row-major FP64 array (ld even, base
// 16-byte aligned), in place.  ipiv (device, n int32) gets absolute pivot rows; perm (device,
// n int32, may be null) gets the final row permutation; status[kInfo] = 1 on a singular pivot.
int32_t lu_factor_f64(Ctx* ctx, cudaStream_t st, double* A, int64_t ld, int64_t n, int32_t* ipiv, int32_t* perm);

// Solves A X = B from the factors of lu_factor_f64: B (n x nrhs, row stride ldb elements) is
// overwritten with X.  perm is the permutation from lu_factor_f64.
// `tmp` (n x ldb doubles) is the gather buffer; when null the context workspace is used.
int32_t lu_solve_f64(Ctx* ctx, cudaStream_t st, const double* LU, int64_t ld, int64_t n, const int32_t* perm,
                     double* B, int64_t ldb, int64_t nrhs, double* tmp = nullptr);

// Blocked FP64 triangular solve of X (n x nrhs, row stride ldx) in place with a triangle of the FP64
// LU factors: kTriL unit-lower L, kTriU upper U, kTriUt = U^T (lower), kTriLt = L^T (unit upper).
enum TriMode : int { kTriL = 0, kTriU = 1, kTriUt = 2, kTriLt = 3 };
int32_t ensure_side_stream(Ctx* ctx);
// two triangular solves in sequence on the same factors (X <- T2^-1 T1^-1 X); where both run the
// persistent sweep, the diagonal-block inverses and coupling blocks of the second are formed on
// the side stream while the first's are formed and swept
int32_t tri_solve2_f64(Ctx* ctx, cudaStream_t st, const double* LU, int64_t ld, int64_t n, int mode1, int mode2,
                       double* X, int64_t ldx, int64_t nrhs);
int32_t tri_solve_f64(Ctx* ctx, cudaStream_t st, const double* LU, int64_t ld, int64_t n, int mode, double* X,
                      int64_t ldx, int64_t nrhs);

// Adjoint of the LU solve from the FP64 factors (adjoint.cu): Lambda = A^{-T} G and, when dA is
// non-null, dA = -Lambda X^T (op B2M_DO_NONE) or dA -= Lambda X^T (op B2M_DO_ADD).  Y (n x ldy) is
// scratch for the two triangular sweeps.
int32_t solve_adjoint_f64(Ctx* ctx, cudaStream_t st, const double* LU, int64_t ld, int64_t n, const int32_t* perm,
                          const double* X, int64_t ldx, const double* G, int64_t ldg, int64_t nrhs, double* Lam,
                          int64_t ldl, double* dA, int64_t ldd, int op, double* Y, int64_t ldy);

// C (M x N) op= A (M x K) B (K x N) in FP64 emulated with int8 slices on tcgen05 (ozaki.cu)
int32_t ozaki_gemm(Ctx* ctx, cudaStream_t st, const double* A, int64_t lda, const double* B, int64_t ldb, double* C,
                   int64_t ldc, int64_t M, int64_t N, int64_t K, int op, int s);

// Compares `rows` sampled rows of C (M x N) with the compensated (Dot2) product A B and returns, in
// host_out4, max |C - C*|, max |A||B|, sum (C - C*)^2, sum C*^2 over them (report.cu).  Element
// (m, k) of A is A[m lda + k] when a_kmajor, else A[k lda + m]; (k, n) of B is B[k ldb + n] when
// b_nmajor, else B[n ldb + k].  Synchronizes the stream.
int32_t gemm_error_report(Ctx* ctx, cudaStream_t st, const double* C, int64_t ldc, const double* A, int64_t lda,
                          bool a_kmajor, const double* B, int64_t ldb, bool b_nmajor, int64_t M, int64_t N, int64_t K,
                          int rows, double* host_out4);

// Cholesky (chol.cu).  chol_factor_f64: A = L L^T in place (lower triangle; the strict upper triangle
// is scratch), status[kInfo] = 1 when A is not positive definite.  chol_solve_f64: B <- A^-1 B from
// the factor F (lower, with diagonal), using W (n x ldw) as scratch.  copy_lower: dst's lower
// triangle (with diagonal) <- src's (only when status[kInfo] == 0 if only_if_ok).  split_nr / join_nr:
// between one factor and the Numerical-Recipes form (strict lower triangle + diagonal vector P at
// byte stride lwp).
int32_t chol_factor_f64(Ctx* ctx, cudaStream_t st, double* A, int64_t ld, int64_t n);
int32_t chol_solve_f64(Ctx* ctx, cudaStream_t st, const double* F, int64_t ldf, int64_t n, double* W, int64_t ldw,
                       double* B, int64_t ldb, int64_t nrhs);
int32_t copy_lower(Ctx* ctx, cudaStream_t st, double* dst, int64_t ldd, const double* src, int64_t lds, int64_t n,
                   bool only_if_ok);
int32_t split_nr(Ctx* ctx, cudaStream_t st, double* Lnr, int64_t ldl, double* P, int64_t lwp, const double* F,
                 int64_t ldf, int64_t n);
int32_t join_nr(Ctx* ctx, cudaStream_t st, double* F, int64_t ldf, const double* Lnr, int64_t ldl, const double* P,
                int64_t lwp, int64_t n);

// Complex LU (zlu.cu) on split real / imaginary planes (row stride ld, even, 16-byte aligned):
// zlu_factor in place with the reference's CAbs1 pivot rule (ipiv as the reference's, perm the row
// permutation, may be null); zlu_solve overwrites B (planes, ldb) with X using the factors, perm and
// the scratch planes tre/tim (n x ldb); z_(de)interleave convert between TComplex arrays (byte
// stride) and planes; z_determinant writes (re, im) to d_det2.
int32_t zlu_factor(Ctx* ctx, cudaStream_t st, double* re, double* im, int64_t ld, int64_t n, int32_t* ipiv,
                   int32_t* perm);
int32_t zlu_solve(Ctx* ctx, cudaStream_t st, const double* lre, const double* lim, int64_t ld, int64_t n,
                  const int32_t* perm, double* bre, double* bim, int64_t ldb, int64_t nrhs, double* tre, double* tim);
int32_t z_deinterleave(Ctx* ctx, cudaStream_t st, const double* src, int64_t lws, double* re, double* im, int64_t ld,
                       int64_t rows, int64_t cols);
int32_t z_interleave(Ctx* ctx, cudaStream_t st, double* dst, int64_t lwd, const double* re, const double* im,
                     int64_t ld, int64_t rows, int64_t cols, bool only_if_ok);
int32_t z_determinant(Ctx* ctx, cudaStream_t st, const double* re, const double* im, int64_t ld, int64_t n,
                      const int32_t* ipiv, double* d_det2);

// Builds perm from ipiv on the device (used when factors come from outside: b2m_MatrixLUBackSubst).
int32_t perm_from_ipiv(Ctx* ctx, cudaStream_t st, const int32_t* ipiv, int64_t n, int32_t* perm);

// Determinant from factors: (-1)^{#i: ipiv[i] != i} * prod diag, in the reference's order.
int32_t lu_determinant(Ctx* ctx, cudaStream_t st, const double* LU, int64_t ld, int64_t n, const int32_t* ipiv,
                       double* d_det);

// Factors one m x w panel (w <= 32, row stride ld) with partial pivoting on one thread-block
// cluster; ipiv[col_base + j] = row_base + pivot row.  panel_max_rows: tallest panel supported.
template <typename T>
int32_t launch_panel(Ctx* ctx, cudaStream_t st, T* P, int64_t ld, int m, int w, int row_base, int col_base,
                     int32_t* ipiv);
int panel_max_rows(bool fp64, int w);

// Copies a strided FP64 matrix (rows x cols, byte strides) device to device.
int32_t copy_matrix(Ctx* ctx, cudaStream_t st, double* dst, int64_t ldd_bytes, const double* src, int64_t lds_bytes,
                    int64_t rows, int64_t cols);

}  // namespace b2m

namespace b2m {
// X += R elementwise (rows x cols, strides in elements)
int32_t axpy_matrix(Ctx* ctx, cudaStream_t st, double* X, int64_t ldx, const double* R, int64_t ldr, int64_t rows,
                    int64_t cols);
// *out = B2M_ERR_TIMEOUT if words[kTimeout] != 0, else words[kInfo] (0 leOk, 1 leSingular): the
// result word of the asynchronous device-pointer entry points
int32_t publish_status(Ctx* ctx, cudaStream_t st, const int32_t* words, int32_t* out);
// X[i][i] = v for i < n
int32_t set_diagonal(Ctx* ctx, cudaStream_t st, double* X, int64_t ldx, int64_t n, double v);
// dst = src when status[kInfo] == 0 (strides in elements)
int32_t copy_if_ok(Ctx* ctx, cudaStream_t st, double* dst, int64_t ldd, const double* src, int64_t lds, int64_t rows,
                   int64_t cols);
}  // namespace b2m

namespace b2m {
// K-major FP32 operand for the tensor-core GEMM: rows x cols map of (base, ld) starting at (r0, c0)
struct FOperand {
    const float* base;
    int64_t ld;
    int64_t rows, cols;
    int64_t r0, c0;
};
// C(M x N) op= A(M x K) * Bt(N x K)^T on tcgen05 (split 1 = TF32, 3 = 3xTF32 with lo operands
// laid out exactly like the hi ones).
int32_t sgemm_tc(Ctx* ctx, cudaStream_t st, const FOperand& Ah, const float* Al_base, const FOperand& Bh,
                 const float* Bl_base, float* C, int64_t ldc, int64_t M, int64_t N, int64_t K, int op, int split,
                 bool check_info);
// hi / lo split for 3xTF32 (lo may be null: plain copy), optionally transposing.
int32_t tf32_split(Ctx* ctx, cudaStream_t st, const float* src, int64_t lds, int64_t rows, int64_t cols, float* hi,
                   float* lo, int64_t ldo, bool transpose);

template <typename T>
int32_t launch_swaps(Ctx* ctx, cudaStream_t st, T* A, int64_t ld, int ncols, int c0, int w, const int32_t* ipiv,
                     int32_t* perm);
template <typename T>
int32_t launch_trsm_small(Ctx* ctx, cudaStream_t st, const T* L, int64_t ldl, T* B, int64_t ldb, int k, int ncols,
                          bool upper);
}  // namespace b2m

namespace b2m {
// Batched solves of `count` independent systems (batched.cu); metadata arrays are host memory,
// A/B/X/info/iters device memory.  tune_out (may be null) receives the tile shape used.
int32_t batch_solve(Ctx* ctx, cudaStream_t st, int64_t count, const int32_t* n, const int32_t* k,
                    const int64_t* a_off, const int64_t* b_off, const double* A, const double* B, double* X,
                    int mode, int32_t* info, int32_t* iters, BatchTune* tune_out);
}  // namespace b2m

namespace b2m {
struct MixedReport {
    int32_t iterations;
    int32_t fell_back;
    double backward_error;
    double ir_backward_error;
    double forward_error;  // estimate: last correction over the solution, normwise (inf-norms)
};
// FP32 factorisation of the mixed solve (lu_f32.cu): tournament-pivoting panels, tcgen05
// trailing updates (mode 1 TF32, 3 3xTF32), and the inverses of the kTrsvNB-row diagonal blocks
// of L and U used by the refinement's blocked triangular solves.
constexpr int kTrsvNB = 128;
struct F32Scratch {
    int* cand;
    unsigned* counters;
    size_t counters_bytes;
    float* top;
    float* mvals;
    float* wmat;
    int* moves;
    float* lmul;
    int32_t* pmap;
    float* lpinv;
    float *bth, *btl, *ah, *al;
    float *linv, *uinv;
    float *wl, *wu;  // coupling blocks T_bb^-1 T_{b,b-1} (L) and T_bb^-1 T_{b,b+1} (U)
    unsigned long long* ll;  // published block solutions of the persistent refinement sweeps
};
constexpr int kSweepGroups = 2;  // right-hand-side groups of 8 in one persistent sweep (16 columns)
size_t f32_scratch_bytes(int64_t n);
F32Scratch f32_scratch_carve(void* base, int64_t n);
// A (n x n, row stride ld a multiple of 32, 128-byte aligned) is factored in place as P A = L U;
// perm[i] = original row of factor row i.  status[kInfo] != 0 on a tiny pivot.
int32_t lu_factor_f32(Ctx* ctx, cudaStream_t st, float* A, int64_t ld, int64_t n, int32_t* perm, int mode,
                      const F32Scratch& s);
// A X = B with an FP32 tensor-core factorisation and FP64 refinement to normwise backward error
// <= tol; falls back to the plain FP64 solve when refinement stalls.  Device operands, even strides.
int32_t solve_mixed(Ctx* ctx, cudaStream_t st, const double* A, int64_t lda, int64_t n, const double* B, int64_t ldb,
                    double* X, int64_t ldx, int64_t nrhs, int mode, int max_iter, double tol, MixedReport* rep);
// plain FP64 LU solve of device operands (factors in a workspace); fills rep->backward_error
int32_t solve_plain_f64(Ctx* ctx, cudaStream_t st, const double* A, int64_t lda, int64_t n, const double* B,
                        int64_t ldb, double* X, int64_t ldx, int64_t nrhs, MixedReport* rep);
}  // namespace b2m
