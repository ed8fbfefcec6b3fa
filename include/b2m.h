/*
 * b2m.h -- C ABI of libb2m, the B200 (sm_100a) implementation of mrMath's dense FP64
 * GEMM + partial-pivoting LU path.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, returns an int32 status
 * and never throws.  Conventions are those of the reference (Object Pascal, mikerabat/mrmath):
 *   - matrices are row-major FP64; strides ("LineWidth") are in BYTES;
 *   - width = number of columns, height = number of rows (NativeInt -> int64_t);
 *   - pivot vectors are int32, 0-based, with LAPACK-ipiv meaning: indx[i] is the absolute row
 *     that was swapped with row i at elimination step i (LinAlgLU.pas:120-136, 181-281);
 *   - status 0 = leOk, 1 = leSingular (MatrixConst.pas:28); negative = library errors.
 *
 * Two families:
 *   b2m_Matrix*      host buffers.  Drop-in replacements for the reference routine of the same
 *                    name; data is copied to the device, computed, copied back; synchronous.
 *   b2m_dev_Matrix*  device buffers (device pointers, byte strides), asynchronous on the
 *                    context's stream; results (status, determinant) come back through device
 *                    or host pointers as documented.
 */
#ifndef B2M_H
#define B2M_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status codes */
#define B2M_OK               0   /* leOk */
#define B2M_SINGULAR         1   /* leSingular: |pivot| <= 10/MaxDouble (LinAlgLU.pas:262) */
#define B2M_ERR_DIM         -1   /* dimension / stride error (the reference's 'Dimension error' asserts) */
#define B2M_ERR_CUDA        -2   /* a CUDA call failed; b2m_last_error() has the text */
#define B2M_ERR_ALLOC       -3   /* device or pinned allocation failed */
#define B2M_ERR_TIMEOUT     -4   /* a bounded in-kernel wait gave up (never expected) */
#define B2M_ERR_ARG         -5   /* null pointer / invalid enum */
#define B2M_ERR_NOCONV      -6   /* mixed-precision refinement did not converge and fallback was disabled */
#define B2M_ERR_UNSUPPORTED -7   /* size outside what this build supports */
#define B2M_ERR_FORMAT      -8   /* a file is not a saved TDoubleMatrix stream */

/* destination operation of the blocked multiplication, TMatrixMultDestOperation (MatrixConst.pas:147) */
#define B2M_DO_NONE 0
#define B2M_DO_ADD  1
#define B2M_DO_SUB  2

typedef struct b2m_ctx b2m_ctx;

#if defined(__GNUC__)
#define B2M_API __attribute__((visibility("default")))
#else
#define B2M_API
#endif

/* ------------------------------------------------------------------ context
 * A context owns one device, one stream, the device workspaces and the captured graphs.
 * It is single-threaded; the library is re-entrant across contexts.  There is no counterpart
 * in the reference (its state is global: MatrixASMStubSwitch.pas InitMathFunctions). */
B2M_API int32_t     b2m_create(int32_t device, b2m_ctx** out);
B2M_API int32_t     b2m_destroy(b2m_ctx* ctx);
/* Run subsequent calls on a caller stream (a cudaStream_t; NULL is the legacy default stream). */
B2M_API int32_t     b2m_set_stream(b2m_ctx* ctx, void* stream);
/* Go back to the context's own (non-blocking) stream. */
B2M_API int32_t     b2m_use_own_stream(b2m_ctx* ctx);
/* Launch sequences whose shape depends only on sizes and buffers (factorisations, solves) are
 * captured into CUDA graphs on first use and replayed afterwards (default on); 0 launches
 * every kernel from the host instead. */
B2M_API int32_t     b2m_use_graphs(b2m_ctx* ctx, int32_t enable);
B2M_API int32_t     b2m_synchronize(b2m_ctx* ctx);
/* Progress callback of the LU-based routines, the counterpart of TLinEquProgress
 * (MatrixConst.pas:31, called with numCalc*100 div numCols at LinAlgLU.pas:272-276): `fn(percent,
 * user)` runs on a CUDA host thread after every factored panel of the FP64 LU (every 32, 16 or 8
 * columns), with percent = columns factored * 100 div n, in order.  It must not call CUDA or this
 * library.  While a callback is set, factorisations run without graph replay and a call first
 * waits for the context's previous work.  NULL removes it. */
typedef void (*b2m_progress_fn)(int32_t percent, void* user);
B2M_API int32_t     b2m_set_progress(b2m_ctx* ctx, b2m_progress_fn fn, void* user);
/* ------------------------------------------------------------------ resident matrices
 * Device-resident storage for a matrix class that keeps its data on the GPU across chained calls
 * (Mult, SolveLinEQ, Invert ... on the b2m_dev_* entry points), so that only the first upload and
 * the final download cross PCIe.  No counterpart in the reference, whose TDoubleMatrix owns host
 * memory (Matrix.pas).  A sub-matrix view (SetSubMatrix, Matrix.pas:70) is a pointer into the
 * parent, p + row * (LineWidth / 8) + col, with the parent's LineWidth: every b2m_dev_* entry point
 * takes arbitrary byte strides.
 *   b2m_alloc     rows x cols doubles on the context's device; *LineWidth receives the row stride
 *                 in bytes (padded to 128 bytes).  Free with b2m_free.
 *   b2m_upload / b2m_download  host <-> device copies of rows x cols with byte strides on both
 *                 sides, synchronous (they wait for the context's stream). */
B2M_API int32_t     b2m_alloc(b2m_ctx* ctx, int64_t rows, int64_t cols, double** out, int64_t* LineWidth);
B2M_API int32_t     b2m_free(b2m_ctx* ctx, double* p);
B2M_API int32_t     b2m_upload(b2m_ctx* ctx, double* dst, int64_t dstLineWidth, const double* src,
                               int64_t srcLineWidth, int64_t rows, int64_t cols);
B2M_API int32_t     b2m_download(b2m_ctx* ctx, double* dst, int64_t dstLineWidth, const double* src,
                                 int64_t srcLineWidth, int64_t rows, int64_t cols);
/* ------------------------------------------------------------------ saved matrices
 * The reference's binary persistence format ("RMCLS" streams of TBinaryReaderWriter,
 * BinaryReaderWriter.pas) for TDoubleMatrix objects, the counterpart of ReadObjFromFile
 * (BaseMathPersistence.pas:153) and TDoubleMatrix.SaveToFile(..., TBinaryReaderWriter): matrices a
 * Pascal program saved, and the reference's fixtures (Test/MatrixData1.txt ...), load straight into
 * host or device buffers.  `info` receives the full size and the saved sub-matrix view; with dst NULL
 * the call only queries it.  B2M_ERR_FORMAT: not a saved TDoubleMatrix; B2M_ERR_ARG: no such file. */
typedef struct b2m_matrix_info {
    int64_t width, height;            /* the full matrix that "data" holds, row by row */
    int64_t sub_width, sub_height;    /* the saved sub-matrix view (SetSubMatrix) */
    int64_t offset_x, offset_y;
} b2m_matrix_info;
B2M_API int32_t     b2m_ReadMatrixFile(const char* path, b2m_matrix_info* info, double* dst, int64_t LineWidth);
/* the same into device memory (dst a device pointer, e.g. from b2m_alloc); synchronous */
B2M_API int32_t     b2m_dev_ReadMatrixFile(b2m_ctx* ctx, const char* path, b2m_matrix_info* info, double* dst,
                                           int64_t LineWidth);
/* writes width x height doubles (byte stride LineWidth) as a saved TDoubleMatrix (empty Name, the full
 * matrix as its view), section for section as the reference's saved fixtures */
B2M_API int32_t     b2m_WriteMatrixFile(const char* path, const double* src, int64_t LineWidth, int64_t width,
                                        int64_t height);
/* Number of polls after which a bounded wait of the mixed solve's refinement sweeps gives up
 * (polls < 0 restores the built-in limit, about a second of spinning).  No counterpart in the
 * reference: a lower limit exists to exercise the timeout path -- with 0 polls every dependent
 * wait gives up at once, the call returns B2M_ERR_TIMEOUT and the context stays usable. */
B2M_API int32_t     b2m_set_wait_limit(b2m_ctx* ctx, int64_t polls);
B2M_API const char* b2m_last_error(b2m_ctx* ctx);
B2M_API const char* b2m_status_string(int32_t status);
/* Number of kernels this context has launched so far (device work accounting). */
B2M_API int64_t     b2m_kernel_launches(b2m_ctx* ctx);
/* Execution facts of this context (no counterpart in the reference): B2M_INFO_NUM_SMS, the
 * device's SM count; B2M_INFO_SWEEP_CTAS, the co-resident CTAs of the refinement sweep (-1 before
 * the first mixed solve); B2M_INFO_CHAIN_CLUSTERS, the co-resident 8-CTA clusters of the chained
 * sweep (0: not usable here, -1: not probed yet); B2M_INFO_CHAIN_PROBE, why the chained sweep is not
 * used (0 it is, 1 shared-memory attribute refused, 2 occupancy query failed, 3 launch failed, 4 no
 * cluster fits) times 1000 plus the CUDA error code. */
#define B2M_INFO_NUM_SMS        1
#define B2M_INFO_SWEEP_CTAS     2
#define B2M_INFO_CHAIN_CLUSTERS 3
#define B2M_INFO_CHAIN_PROBE    4
#define B2M_INFO_CHAIN_CLUSTERS4 5  /* the same as B2M_INFO_CHAIN_CLUSTERS for 4-CTA clusters */
#define B2M_INFO_BATCH_BIG_WARPS 6  /* warps per system of order > small_n in the tile shape chosen for
                                       the last batch plan (8: a whole CTA, 4: two systems per CTA;
                                       0 before any batch) */
B2M_API int32_t     b2m_ctx_info(b2m_ctx* ctx, int32_t what, int64_t* value);
/* Event profiler: when enabled, every launch is bracketed by CUDA events on its own stream and
 * its algorithmic work is recorded per kernel class (0 FP64 GEMM, 1 panel, 2 row swaps,
 * 3 triangular solve, 4 tensor-core GEMM, 5 solve/refinement kernels, 6 other, e.g. the FP64
 * residual).  Work is FLOPs for classes 0 and 4 and HBM bytes for the others.  Enabling (or
 * disabling) resets the counters.  Reading synchronizes the device. */
B2M_API int32_t     b2m_profile(b2m_ctx* ctx, int32_t enable);
B2M_API int32_t     b2m_profile_read(b2m_ctx* ctx, int32_t kernel_class, int64_t* launches, double* ms,
                                     double* work);

/* ------------------------------------------------------------------ GEMM
 * Replaces MatrixMult / MatrixMultEx (MatrixASMStubSwitch.pas:769-782),
 * MatrixMultT1 / MatrixMultT1Ex (:812-823) and MatrixMultT2 / MatrixMultT2Ex (:853-863).
 * trans 0: dest(height1 x width2)  op=  mt1(height1 x width1)   * mt2(height2 x width2), width1 = height2
 * trans 1: dest(width1  x width2)  op=  mt1(height1 x width1)^T * mt2(height2 x width2), height1 = height2
 * trans 2: dest(height1 x height2) op=  mt1(height1 x width1)   * mt2(height2 x width2)^T, width1 = width2
 * op: B2M_DO_NONE (dest =), B2M_DO_ADD (dest +=), B2M_DO_SUB (dest -=). */
B2M_API int32_t b2m_MatrixMultEx(b2m_ctx* ctx, double* dest, int64_t destLineWidth, const double* mt1, const double* mt2,
                         int64_t width1, int64_t height1, int64_t width2, int64_t height2,
                         int64_t LineWidth1, int64_t LineWidth2, int32_t op, int32_t trans);
B2M_API int32_t b2m_dev_MatrixMultEx(b2m_ctx* ctx, double* dest, int64_t destLineWidth, const double* mt1,
                             const double* mt2, int64_t width1, int64_t height1, int64_t width2, int64_t height2,
                             int64_t LineWidth1, int64_t LineWidth2, int32_t op, int32_t trans);
/* MatrixMultEx (trans 0) emulated on the INT8 tensor cores (Ozaki scheme).  No counterpart in the
 * reference: an alternative engine for MatrixMult / MatrixMultEx (MatrixASMStubSwitch.pas:769-782),
 * same arguments plus `slices` (2..10, 0 = 8): every row of mt1 and column of mt2 is scaled by a
 * power of two and cut into `slices` signed 7-bit pieces, and the pairwise products are summed
 * exactly in int32 and scaled in FP64.  The error is below about 2^-7(slices+1) times
 * |row max of mt1| |column max of mt2| times the inner dimension. */
B2M_API int32_t b2m_MatrixMultOzaki(b2m_ctx* ctx, double* dest, int64_t destLineWidth, const double* mt1,
                            const double* mt2, int64_t width1, int64_t height1, int64_t width2, int64_t height2,
                            int64_t LineWidth1, int64_t LineWidth2, int32_t op, int32_t slices);
B2M_API int32_t b2m_dev_MatrixMultOzaki(b2m_ctx* ctx, double* dest, int64_t destLineWidth, const double* mt1,
                                const double* mt2, int64_t width1, int64_t height1, int64_t width2,
                                int64_t height2, int64_t LineWidth1, int64_t LineWidth2, int32_t op, int32_t slices);

/* Error report of a product.  No counterpart in the reference (MatrixMult returns only the product):
 * `sample_rows` rows of dest (spread evenly; <= 0 means 16) are compared with op(mt1) op(mt2)
 * computed with the compensated dot product Dot2 (Ogita, Rump, Oishi 2005; as accurate as twice
 * the working precision).  dest must hold a B2M_DO_NONE result of b2m_MatrixMultEx (any trans) or
 * b2m_MatrixMultOzaki (trans 0); arguments as b2m_MatrixMultEx. */
typedef struct b2m_gemm_report {
    int32_t rows_checked;
    int32_t reserved;
    double  forward_error;   /* max |C - C*| / max (|A||B|) over the sampled rows, C* the Dot2 product */
    double  relative_error;  /* ||C - C*||_F / ||C*||_F over the sampled rows */
    double  bound;           /* K 2^-53: the a-priori bound of an FP64 product on the forward_error scale */
} b2m_gemm_report;
B2M_API int32_t b2m_MatrixMultErrorReport(b2m_ctx* ctx, const double* dest, int64_t destLineWidth, const double* mt1,
                                          const double* mt2, int64_t width1, int64_t height1, int64_t width2,
                                          int64_t height2, int64_t LineWidth1, int64_t LineWidth2, int32_t trans,
                                          int32_t sample_rows, b2m_gemm_report* report);
/* device twin: dest, mt1, mt2 device memory; the report is host memory (the call synchronizes) */
B2M_API int32_t b2m_dev_MatrixMultErrorReport(b2m_ctx* ctx, const double* dest, int64_t destLineWidth,
                                              const double* mt1, const double* mt2, int64_t width1, int64_t height1,
                                              int64_t width2, int64_t height2, int64_t LineWidth1,
                                              int64_t LineWidth2, int32_t trans, int32_t sample_rows,
                                              b2m_gemm_report* report);

/* ------------------------------------------------------------------ LU (src/LinAlgLU.pas)
 * Orders up to 32768 (the FP64 pivot panel is held on chip by one 16-CTA cluster, 8 columns wide at
 * the largest orders); larger orders return B2M_ERR_UNSUPPORTED.  The reference has no such limit. */
/* MatrixLUDecompInPlace LinAlgLU.pas:283-295 */
B2M_API int32_t b2m_MatrixLUDecompInPlace(b2m_ctx* ctx, double* A, int64_t LineWidthA, int64_t width, int32_t* indx);
/* MatrixLUDecomp LinAlgLU.pas:297-305 (A is left untouched) */
B2M_API int32_t b2m_MatrixLUDecomp(b2m_ctx* ctx, const double* A, int64_t LineWidthA, double* LUDecomp,
                           int64_t LineWidthLU, int64_t width, int32_t* indx);
/* MatrixLUBackSubst LinAlgLU.pas:315-385, generalised to nrhs columns of B (nrhs = 1 is the reference call). */
B2M_API int32_t b2m_MatrixLUBackSubst(b2m_ctx* ctx, const double* LUDecomp, int64_t LineWidthLU, int64_t width,
                              const int32_t* indx, double* B, int64_t LineWidthB, int64_t nrhs);
/* MatrixInverseInPlace LinAlgLU.pas:388-431 */
B2M_API int32_t b2m_MatrixInverseInPlace(b2m_ctx* ctx, double* A, int64_t LineWidthA, int64_t width);
/* MatrixDeterminant LinAlgLU.pas:433-479 (0 for a singular matrix, status still B2M_OK like the reference) */
B2M_API int32_t b2m_MatrixDeterminant(b2m_ctx* ctx, const double* A, int64_t LineWidthA, int64_t width, double* det);
/* MatrixLinEQSolve LinAlgLU.pas:481-592.  NumRefinements > 0 runs the reference's fixed-count FP64
   refinement (residual A*x - b, back-substitution, x -= d), each column reading x along its column. */
B2M_API int32_t b2m_MatrixLinEQSolve(b2m_ctx* ctx, const double* A, int64_t LineWidthA, int64_t width, const double* B,
                             int64_t LineWidthB, double* X, int64_t LineWidthX, int64_t Width2,
                             int64_t NumRefinements);

/* device-resident twins (device pointers; indx / det / status are device pointers too).  The
 * device result word *status (may be NULL) receives 0 (leOk), 1 (leSingular) or B2M_ERR_TIMEOUT
 * when a bounded in-kernel wait gave up and the outputs are unfinished. */
B2M_API int32_t b2m_dev_MatrixLUDecompInPlace(b2m_ctx* ctx, double* A, int64_t LineWidthA, int64_t width, int32_t* indx,
                                      int32_t* status);
B2M_API int32_t b2m_dev_MatrixLUBackSubst(b2m_ctx* ctx, const double* LUDecomp, int64_t LineWidthLU, int64_t width,
                                  const int32_t* indx, double* B, int64_t LineWidthB, int64_t nrhs);
B2M_API int32_t b2m_dev_MatrixLinEQSolve(b2m_ctx* ctx, const double* A, int64_t LineWidthA, int64_t width,
                                 const double* B, int64_t LineWidthB, double* X, int64_t LineWidthX,
                                 int64_t Width2, int64_t NumRefinements, int32_t* status);
B2M_API int32_t b2m_dev_MatrixInverseInPlace(b2m_ctx* ctx, double* A, int64_t LineWidthA, int64_t width, int32_t* status);
B2M_API int32_t b2m_dev_MatrixDeterminant(b2m_ctx* ctx, const double* A, int64_t LineWidthA, int64_t width, double* det);

/* ------------------------------------------------------------------ complex LU (LinAlgLU.pas:1147-1603)
 * TComplex matrices: interleaved (real, imag) doubles, 16 bytes per element, strides in bytes.
 * Pivoting as the reference's complex leaf: largest |re| + |im| (CAbs1), first maximum wins,
 * singular when it is <= 10/MaxDouble; the column is scaled by CInv(pivot); back substitution
 * divides by U's diagonal with CDiv (Smith's formula). */
/* CplxMatrixLUDecompInPlace LinAlgLU.pas:1308-1320 */
B2M_API int32_t b2m_CplxMatrixLUDecompInPlace(b2m_ctx* ctx, double* A, int64_t LineWidthA, int64_t width,
                                              int32_t* indx);
/* CplxMatrixLUBackSubst LinAlgLU.pas:1322-1391, generalised to nrhs columns of B */
B2M_API int32_t b2m_CplxMatrixLUBackSubst(b2m_ctx* ctx, const double* LUDecomp, int64_t LineWidthLU, int64_t width,
                                          const int32_t* indx, double* B, int64_t LineWidthB, int64_t nrhs);
/* CplxMatrixLinEQSolve LinAlgLU.pas:1393-1508 (no refinement: the reference's refinement branch
 * calls the real back substitution on complex data and is not reproduced) */
B2M_API int32_t b2m_CplxMatrixLinEQSolve(b2m_ctx* ctx, const double* A, int64_t LineWidthA, int64_t width,
                                         const double* B, int64_t LineWidthB, double* X, int64_t LineWidthX,
                                         int64_t Width2);
/* CplxMatrixInverseInPlace LinAlgLU.pas:1510-1552 (A untouched when singular) */
B2M_API int32_t b2m_CplxMatrixInverseInPlace(b2m_ctx* ctx, double* A, int64_t LineWidthA, int64_t width);
/* CplxMatrixDeterminant LinAlgLU.pas:1554-1603: det[0] = real, det[1] = imag; (0, 0) for a singular
 * matrix with status B2M_OK */
B2M_API int32_t b2m_CplxMatrixDeterminant(b2m_ctx* ctx, const double* A, int64_t LineWidthA, int64_t width,
                                          double* det);

/* ------------------------------------------------------------------ Cholesky (src/LinAlgCholesky.pas)
 * Results: 0 = crOk, 1 = crNoPositiveDefinite (TCholeskyResult, MatrixConst.pas:30): a diagonal
 * element <= 0 or NaN before its square root; A is then left unchanged. */
/* MatrixCholeskyInPlace4 LinAlgCholesky.pas:106-123 (the routine of TDoubleMatrix.Cholesky,
 * DblMatrix.pas:967-990): A = L L^T with L in the lower triangle of A (diagonal included); the strict
 * upper triangle is not written.  pnlSize (0 = 32) is accepted for the reference's signature; the
 * device blocking is the library's own. */
B2M_API int32_t b2m_MatrixCholeskyInPlace4(b2m_ctx* ctx, double* A, int64_t LineWidthA, int64_t width,
                                           int64_t pnlSize);
B2M_API int32_t b2m_dev_MatrixCholeskyInPlace4(b2m_ctx* ctx, double* A, int64_t LineWidthA, int64_t width,
                                               int32_t* status);
/* MatrixCholeskyInPlace LinAlgCholesky.pas:270-332 (Numerical-Recipes form): L strictly below the
 * diagonal of A, its diagonal in P (element i at byte offset i * LineWidthP); A's diagonal and upper
 * triangle are not written. */
B2M_API int32_t b2m_MatrixCholeskyInPlace(b2m_ctx* ctx, double* A, int64_t LineWidthA, int64_t width, double* P,
                                          int64_t LineWidthP);
/* MatrixCholeskySolveLinEq LinAlgCholesky.pas:352-421, generalised to nrhs columns: A X = B from the
 * factor of b2m_MatrixCholeskyInPlace (P not NULL: L below A's diagonal, diagonal in P) or of
 * b2m_MatrixCholeskyInPlace4 (P NULL: diagonal on A's diagonal).  Only the lower triangle is read. */
B2M_API int32_t b2m_MatrixCholeskySolveLinEq(b2m_ctx* ctx, const double* A, int64_t LineWidthA, int64_t width,
                                             const double* P, int64_t LineWidthP, const double* B, int64_t LineWidthB,
                                             double* X, int64_t LineWidthX, int64_t nrhs);
B2M_API int32_t b2m_dev_MatrixCholeskySolveLinEq(b2m_ctx* ctx, const double* A, int64_t LineWidthA, int64_t width,
                                                 const double* P, int64_t LineWidthP, const double* B,
                                                 int64_t LineWidthB, double* X, int64_t LineWidthX, int64_t nrhs);

/* ------------------------------------------------------------------ mixed-precision solve
 * No counterpart in the reference.  A X = B with an FP32 LU whose trailing and triangular-solve
 * updates run on the tcgen05 tensor cores (mode B2M_MIXED_TF32: TF32; B2M_MIXED_3XTF32: hi/lo
 * split, about FP32 accuracy), refined in FP64 (residual B - A X, update, normwise backward-error
 * stopping test) until max_j ||b_j - A x_j||_inf / (||A||_inf ||x_j||_inf + ||b_j||_inf) <= tol
 * (tol <= 0 means n * 2^-53; maxIter <= 0 means 30 for TF32, 10 for 3xTF32).  When refinement stalls, the plain FP64 LU solve runs instead and
 * report->fell_back = 1.  Status as b2m_MatrixLinEQSolve. */
#define B2M_MIXED_TF32   1
#define B2M_MIXED_3XTF32 3
typedef struct b2m_solve_report {
    int32_t iterations;      /* refinement steps taken */
    int32_t fell_back;       /* 1 if the plain FP64 solve produced X */
    double  backward_error;  /* normwise backward error of the returned X (FP64 residual) */
    double  refinement_backward_error;  /* the last refinement step's, before any fallback */
    double  forward_error;   /* normwise forward-error estimate of ||x - x*|| / ||x*|| (max over columns j,
                                inf-norms).  Refinement: ||d_j|| rho_j / ||x_j|| with d the last
                                correction applied and rho_j = ||d_j|| / ||d_j of the step before|| (the
                                observed contraction; 1 after a single step).  Fallback: ||d_j|| / ||x_j||
                                with d one extra correction computed with the FP64 factors. */
} b2m_solve_report;
B2M_API int32_t b2m_MatrixLinEQSolveMixed(b2m_ctx* ctx, const double* A, int64_t LineWidthA, int64_t width,
                                          const double* B, int64_t LineWidthB, double* X, int64_t LineWidthX,
                                          int64_t Width2, int32_t mode, int32_t maxIter, double tol,
                                          b2m_solve_report* report);
B2M_API int32_t b2m_dev_MatrixLinEQSolveMixed(b2m_ctx* ctx, const double* A, int64_t LineWidthA, int64_t width,
                                              const double* B, int64_t LineWidthB, double* X, int64_t LineWidthX,
                                              int64_t Width2, int32_t mode, int32_t maxIter, double tol,
                                              b2m_solve_report* report);

/* SolveLinEQAdjoint.  No counterpart in the reference: the adjoint (reverse-mode derivative) of
 * MatrixLinEQSolve (LinAlgLU.pas:481-592).  From the factors of b2m_MatrixLUDecomp (LUDecomp and the
 * reference-format interchange vector indx), the solution X (width x nrhs) of A X = B and a seed
 * G = dLoss/dX, computes Lambda = A^{-T} G (= dLoss/dB) and, when dA is not NULL, the rank-nrhs
 * update dA = -Lambda X^T (op B2M_DO_NONE) or dA -= Lambda X^T (op B2M_DO_ADD, to accumulate).
 * Strides in bytes. */
B2M_API int32_t b2m_MatrixLinEQSolveAdjoint(b2m_ctx* ctx, const double* LUDecomp, int64_t LineWidthLU, int64_t width,
                                    const int32_t* indx, const double* X, int64_t LineWidthX, const double* G,
                                    int64_t LineWidthG, int64_t nrhs, double* Lambda, int64_t LineWidthLambda,
                                    double* dA, int64_t LineWidthdA, int32_t op);
/* Device twin: every pointer is device memory (indx as produced by b2m_dev_MatrixLUDecompInPlace);
 * asynchronous on the context's stream. */
B2M_API int32_t b2m_dev_MatrixLinEQSolveAdjoint(b2m_ctx* ctx, const double* LUDecomp, int64_t LineWidthLU,
                                        int64_t width, const int32_t* indx, const double* X, int64_t LineWidthX,
                                        const double* G, int64_t LineWidthG, int64_t nrhs, double* Lambda,
                                        int64_t LineWidthLambda, double* dA, int64_t LineWidthdA, int32_t op);

/* Batched solves of many independent systems of uneven order in one persistent launch.  No
 * counterpart in the reference, which solves one system per MatrixLinEQSolve call
 * (LinAlgLU.pas:481-592); each system follows that routine's pivoting, singularity test and
 * substitution.  System i has order n[i] (1..256) and nrhs[i] (1..8) right-hand sides; A_i is
 * row-major n_i x n_i at A + a_off[i], B_i and X_i are row-major n_i x nrhs_i at B + b_off[i] and
 * X + b_off[i] (offsets in doubles).  The plan arrays n, nrhs, a_off, b_off are host memory.
 * mode 0: FP64 LU with partial pivoting; mode 1: FP32 factorisation + FP64 refinement to
 * backward error <= n_i 2^-53, refactored in FP64 when refinement stalls.  info[i] = 0 (leOk) or
 * 1 (leSingular); iters[i] (may be NULL) = refinement steps in mode 1, -1 when FP64 was needed.
 * The first call with a new plan runs the autotuner (it times the candidate tile shapes). */
B2M_API int32_t b2m_BatchLinEQSolve(b2m_ctx* ctx, int64_t count, const int32_t* n, const int32_t* nrhs,
                                    const int64_t* a_off, const int64_t* b_off, const double* A, const double* B,
                                    double* X, int32_t mode, int32_t* info, int32_t* iters);
/* Device twin: A, B, X, info, iters are device memory (the plan arrays stay on the host);
 * asynchronous on the context's stream, replayed from a CUDA graph after the first call. */
B2M_API int32_t b2m_dev_BatchLinEQSolve(b2m_ctx* ctx, int64_t count, const int32_t* n, const int32_t* nrhs,
                                        const int64_t* a_off, const int64_t* b_off, const double* A,
                                        const double* B, double* X, int32_t mode, int32_t* info, int32_t* iters);
/* The autotuner's table, persisted: b2m_batch_tune_save writes every tuned plan (plan signature and
 * its tile shape) to a text file; b2m_batch_tune_load merges such a file into the context, so that a
 * later process skips the timing of the candidate shapes for those plans (*loaded = plans taken;
 * lines with shapes the kernel does not have are skipped; B2M_ERR_FORMAT if the file is not a
 * table).  The reference tunes its block sizes at start-up and keeps nothing
 * (BlockSizeSetup.pas:169-297); this is the persisted form of that step. */
B2M_API int32_t b2m_batch_tune_save(b2m_ctx* ctx, const char* path);
B2M_API int32_t b2m_batch_tune_load(b2m_ctx* ctx, const char* path, int32_t* loaded);
/* The tile shape the autotuner chose for the last batch plan. */
B2M_API int32_t b2m_batch_tune_read(b2m_ctx* ctx, int32_t* small_n, int32_t* group_warps, int32_t* pw_large,
                                    int32_t* pw_small, float* ms);

/* Allocation-free solve.  No counterpart in the reference: it exists for callers that may not
 * allocate device memory (a host program whose memory manager owns all device allocations and
 * forbids any other cudaMalloc, a real-time loop with a fixed memory budget).  Same arguments and
 * result as b2m_dev_MatrixLinEQSolve without refinement, on the given cudaStream_t (NULL = legacy
 * default stream) of the calling thread's current device.  All intermediates live in one static
 * device array of about 2.5 MiB that every GPU loading the library holds until exit; orders up to
 * 512 and up to 64 right-hand sides are accepted, larger sizes return B2M_ERR_UNSUPPORTED.  The
 * first call on a device looks up the array's address (cudaGetSymbolAddress), so make that first
 * call before any stream capture.  Every call shares the array and it keeps the last call's
 * contents: calls that overlap on the GPU (other streams, other host threads) race.  *status
 * (device int32, may be NULL) receives 0 (leOk), 1 (leSingular) or B2M_ERR_TIMEOUT when a bounded
 * wait in the factorisation gave up (X is then unfinished).  The array's address is looked up once
 * per device ordinal and kept: do not use this entry point across a cudaDeviceReset. */
B2M_API int32_t b2m_dev_MatrixLinEQSolveNoAlloc(void* stream, const double* A, int64_t LineWidthA, int64_t width,
                                                const double* B, int64_t LineWidthB, double* X, int64_t LineWidthX,
                                                int64_t Width2, int32_t* status);

#ifdef __cplusplus
}
#endif
#endif /* B2M_H */
