/*
 * mrmath_oracle.h -- CPU restatement of mrMath's dense FP64 GEMM + pivoted-LU path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA product
 * (libb2m) is compared against, and the CPU baseline that bench.py times beside it.
 * Nothing in the product path links, loads or calls it.
 *
 * Every routine restates one routine of the reference (Object Pascal, mikerabat/mrmath);
 * the reference file:line is given beside each declaration.  Conventions follow the
 * reference exactly: row-major FP64, strides ("LineWidth") in BYTES, pivot vectors int32,
 * sizes int64 (NativeInt), result codes 0 = leOk, 1 = leSingular (MatrixConst.pas:28).
 *
 * Pinning: the MT19937 generator is pinned byte-for-byte to Test/marsenneTwistOrig.txt;
 * the LU / back-substitution / inverse / determinant / GEMM routines are pinned to the
 * known-answer tests of Test/TestLineEquations.pas, Test/TestSimpleMatrixOperations.pas,
 * Test/TestFMA.pas and Test/TestMatrixClass.pas (see tests/test_oracle_kat.py).  No large-n
 * golden output exists in the reference, so large-n agreement is pinned only through those
 * kernels plus cross-implementation tests (single-threaded vs threaded, as the reference does).
 */
#ifndef MRMATH_ORACLE_H
#define MRMATH_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- random engine (src/RandomEng.pas) ---------------- */
typedef struct orc_rng {
    uint32_t mt[624];
    int32_t  mti;          /* fMTi, 625 = "not initialised" as in SetRandMethod (RandomEng.pas:401-402) */
    int32_t  gauss_flag;   /* fRandGFlag */
    double   gauss2;       /* fRandG2 */
} orc_rng;

void     orc_rng_init(orc_rng* r, int32_t seed);                              /* InitMersenne RandomEng.pas:626-644 */
void     orc_rng_init_by_array(orc_rng* r, const uint32_t* key, int32_t len); /* InitMersenneByArr :646-692 */
uint32_t orc_rng_u32(orc_rng* r);                                             /* RandMersenneDblWord :694-731 */
uint32_t orc_rng_lw(orc_rng* r, uint32_t range);                              /* RandMersenneLW (y mod range) */
double   orc_rng_dbl(orc_rng* r);                                             /* RandMersenneDbl :749-765 */
double   orc_rng_gauss(orc_rng* r);                                           /* RandGauss (Marsaglia polar) :283-307 */
/* Row-major fills in the order TDoubleMatrix.InitRandom / MatrixFunc visit elements
   (DblMatrix.pas:2751-2759): uniform [0,1) and Gaussian. */
void     orc_fill_uniform(orc_rng* r, double* dst, int64_t count);
void     orc_fill_gauss(orc_rng* r, double* dst, int64_t count);
/* C3 GEMM inputs: g*2^e, all g = RandGauss first, then all e = RandLW(17) - 8, row-major. */
void     orc_fill_gauss_exp(orc_rng* r, double* dst, int64_t count);

/* ---------------- kernel family (MatrixASMStubSwitch.pas InitMathFunctions) ---------------- */
/* 0 = generic Pascal kernels (SimpleMatrixOperations.pas), 1 = FMA kernels (default itFMA). */
void    orc_set_mode(int32_t mode);
int32_t orc_get_mode(void);

/* ---------------- GEMM ---------------- */
/* dest(h1 x w2) = mt1(h1 x w1) * mt2(h2 x w2), MatrixMult MatrixASMStubSwitch.pas:769-776 */
void orc_matrix_mult(double* dest, int64_t lwd, const double* mt1, const double* mt2,
                     int64_t w1, int64_t h1, int64_t w2, int64_t h2, int64_t lw1, int64_t lw2);
/* BlockMatrixMultiplication BlockedMult.pas:350-474; op 0 doNone, 1 doAdd, 2 doSub */
void orc_block_mult(double* dest, int64_t lwd, const double* mt1, const double* mt2,
                    int64_t w1, int64_t h1, int64_t w2, int64_t h2, int64_t lw1, int64_t lw2,
                    int64_t blockSize, int32_t op);
/* BlockMatrixMultiplicationT1 BlockedMult.pas:477-593: dest(w1 x w2) = mt1^T * mt2 */
void orc_block_mult_t1(double* dest, int64_t lwd, const double* mt1, const double* mt2,
                       int64_t w1, int64_t h1, int64_t w2, int64_t h2, int64_t lw1, int64_t lw2,
                       int64_t blockSize, int32_t op);
/* BlockMatrixMultiplicationT2 BlockedMult.pas:596-724: dest(h1 x h2) = mt1 * mt2^T */
void orc_block_mult_t2(double* dest, int64_t lwd, const double* mt1, const double* mt2,
                       int64_t w1, int64_t h1, int64_t w2, int64_t h2, int64_t lw1, int64_t lw2,
                       int64_t blockSize, int32_t op);
/* GenericMtxMult SimpleMatrixOperations.pas:1561-1591 */
void orc_generic_mult(double* dest, int64_t lwd, const double* mt1, const double* mt2,
                      int64_t w1, int64_t h1, int64_t w2, int64_t h2, int64_t lw1, int64_t lw2);

/* ---------------- LU path (src/LinAlgLU.pas) ---------------- */
int32_t orc_lu_decomp_inplace(double* A, int64_t lwA, int64_t width, int32_t* indx);   /* :283-295 */
int32_t orc_lu_decomp(const double* A, int64_t lwA, double* LU, int64_t lwLU,
                      int64_t width, int32_t* indx);                                  /* :297-305 */
void    orc_lu_backsubst(const double* LU, int64_t lwLU, int64_t width, const int32_t* indx,
                         double* B, int64_t lwB);                                     /* :315-385 */
int32_t orc_inverse_inplace(double* A, int64_t lwA, int64_t width);                   /* :388-431 */
double  orc_determinant(const double* A, int64_t lwA, int64_t width);                 /* :433-479 */
/* MatrixLinEQSolve :481-592.  row_quirk != 0 reproduces the refinement residual that walks x
   along a row (:567); row_quirk == 0 reads x along its column (the evident intent). */
int32_t orc_lineq_solve(const double* A, int64_t lwA, int64_t width, const double* B, int64_t lwB,
                        double* X, int64_t lwX, int64_t width2, int64_t numRefinements, int32_t row_quirk);

/* ---------------- threaded twins = CPU baseline (LinAlgLU.pas:594-1128) ---------------- */
void    orc_set_num_threads(int32_t n);     /* numUseCPUCores, MtxThreadPool.pas:74 */
int32_t orc_get_num_threads(void);
void    orc_thr_matrix_mult(double* dest, int64_t lwd, const double* mt1, const double* mt2,
                            int64_t w1, int64_t h1, int64_t w2, int64_t h2, int64_t lw1, int64_t lw2,
                            int64_t blockSize, int32_t op);                           /* ThrMatrixMultEx2 ThreadedMatrixOperations.pas:612-718 */
int32_t orc_thr_lu_decomp(double* A, int64_t lwA, int64_t width, int32_t* indx);        /* ThrMatrixLUDecomp :788-803 */
int32_t orc_thr_lineq_solve(const double* A, int64_t lwA, int64_t width, const double* B, int64_t lwB,
                            double* X, int64_t lwX, int64_t width2, int64_t numRefinements); /* :986-1128 */
int32_t orc_thr_inverse(double* A, int64_t lwA, int64_t width);                       /* :853-929 */
double  orc_thr_determinant(const double* A, int64_t lwA, int64_t width);             /* :931-984 */

/* ---------------- diagnostics and compensated arithmetic ---------------- */
/* Runs the single-threaded LU on a copy and returns the smallest relative gap
   (|best| - |second|) / |best| seen over all pivot searches (1.0 when a column has one row). */
double  orc_lu_min_pivot_gap(const double* A, int64_t lwA, int64_t width);
/* Ogita-Rump-Oishi Dot2: r = b - A*x for nrhs columns, accurate to ~u^2 cond.  Strides in bytes. */
void    orc_residual_dot2(const double* A, int64_t lwA, int64_t n, const double* X, int64_t lwX,
                          const double* B, int64_t lwB, int64_t nrhs, double* R, int64_t lwR);
/* Normwise backward error per column: max_j ||b_j - A x_j||_inf / (||A||_inf ||x_j||_inf + ||b_j||_inf),
   residual in Dot2. */
double  orc_backward_error(const double* A, int64_t lwA, int64_t n, const double* X, int64_t lwX,
                           const double* B, int64_t lwB, int64_t nrhs);
/* Rows [r0, r0+nr) of C = A*B with every entry a Dot2 dot product (reference entries for GEMM
   forward errors).  Also returns the same rows of |A|*|B| in absAB if non-null. */
void    orc_gemm_rows_dot2(const double* A, int64_t lwA, const double* B, int64_t lwB,
                           int64_t m, int64_t n, int64_t k, int64_t r0, int64_t nr,
                           double* C, int64_t lwC, double* absAB, int64_t lwAbs);

/* ---- complex LU (LinAlgLU.pas:1147-1603): interleaved (real, imag) doubles, strides in bytes */
int32_t orc_cplx_lu_decomp_inplace(double* A, int64_t lwA, int64_t width, int32_t* indx);  /* :1308-1320 */
void    orc_cplx_lu_backsubst(const double* LU, int64_t lwLU, int64_t width, const int32_t* indx, double* B,
                              int64_t lwB);                                                /* :1322-1391 */
int32_t orc_cplx_lineq_solve(const double* A, int64_t lwA, int64_t width, const double* B, int64_t lwB,
                             double* X, int64_t lwX, int64_t nrhs);                        /* :1393-1508 */
int32_t orc_cplx_inverse_inplace(double* A, int64_t lwA, int64_t width);                  /* :1510-1552 */
void    orc_cplx_determinant(const double* A, int64_t lwA, int64_t width, double* det);   /* :1554-1603 */

/* ---- Cholesky (LinAlgCholesky.pas); results 0 = crOk, 1 = crNoPositiveDefinite (MatrixConst.pas:30) */
int32_t orc_cholesky_inplace4(double* A, int64_t lwA, int64_t width, int64_t pnl);   /* :106-123, :54-103 */
int32_t orc_cholesky_inplace2(double* A, int64_t lwA, int64_t width);                /* :205-250 */
int32_t orc_cholesky_nr(double* A, int64_t lwA, int64_t width, double* P, int64_t lwP); /* :270-332 */
void    orc_cholesky_solve_nr(const double* A, int64_t lwA, int64_t width, const double* P, int64_t lwP,
                              const double* B, int64_t lwB, double* X, int64_t lwX);   /* :352-421 */

#ifdef __cplusplus
}
#endif
#endif
