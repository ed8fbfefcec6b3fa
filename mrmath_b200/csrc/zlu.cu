// zlu.cu -- complex (TComplex) LU with partial pivoting, back substitution, solve, inverse and
// determinant on the FP64 building blocks of the real LU.
//
// Reference: InternalRecursiveCplxMatrixLUDecompInPlace (LinAlgLU.pas:1202-1306), CplxLUSwap
// (:1183-1200), CplxLUBacksup (:1147-1181), CplxMatrixLUBackSubst (:1322-1391), CplxMatrixLinEQSolve
// (:1393-1508), CplxMatrixInverseInPlace (:1510-1552), CplxMatrixDeterminant (:1554-1603).  The pivot
// rule is the reference leaf's: the largest CAbs1 = |re| + |im| wins, the first (lowest row) among
// equals, the column is singular when that largest CAbs1 is <= 10/MaxDouble; the column is scaled
// by CInv(pivot) (Smith's formula, CplxSimpleMatrixOperations.pas:288-303) and the pivot placed as
// the reference does; the back substitution divides by U's diagonal with CDiv (:266-285).
//
// B200 design: the interleaved matrix is split into a real and an imaginary plane (row-major, rows
// padded to 128 bytes), so that every complex product of the recursion runs as four real DMMA GEMMs
// (Cr -= Ar Br - Ai Bi, Ci -= Ar Bi + Ai Br), and the row interchanges reuse the real leaf swap
// kernel on each plane.  A 32-column leaf is factored by one 1024-thread CTA (zpanel_kernel) with
// the panel's rows in L2; 32 x 32 unit-lower and upper triangular solves run one warp per four
// right-hand-side columns (lane = row).  The result is interleaved back into the caller's layout.
#include <cfloat>

#include "common.cuh"
#include "kernels.cuh"

namespace b2m {
namespace {

constexpr int kZLeaf = 32;
constexpr int kZPanelThreads = 1024;

struct Planes {
    double* re;
    double* im;
    int64_t ld;
};

__device__ __forceinline__ double2 cinv(double2 x) {
    if (fabs(x.x) >= fabs(x.y)) {
        const double r = x.y / x.x, den = x.x + x.y * r;
        return make_double2(1.0 / den, -r / den);
    }
    const double r = x.x / x.y, den = x.y + r * x.x;
    return make_double2(r / den, -1.0 / den);
}
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
    if (fabs(b.x) >= fabs(b.y)) {
        const double r = b.y / b.x, den = b.x + b.y * r;
        return make_double2((a.x + r * a.y) / den, (a.y - r * a.x) / den);
    }
    const double r = b.x / b.y, den = b.y + b.x * r;
    return make_double2((a.x * r + a.y) / den, (a.y * r - a.x) / den);
}
// x1 - x2 x3 (CSubMul order)
__device__ __forceinline__ double2 csub_mul(double2 x1, double2 x2, double2 x3) {
    return make_double2(x1.x - x2.x * x3.x + x2.y * x3.y, x1.y - x2.x * x3.y - x2.y * x3.x);
}

__global__ void deinterleave_kernel(const double* src, int64_t lws, double* re, double* im, int64_t ld, int64_t rows,
                                    int64_t cols) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= rows * cols) return;
    const int64_t r = e / cols, c = e - r * cols;
    const double2 v = *reinterpret_cast<const double2*>(reinterpret_cast<const char*>(src) + r * lws + c * 16);
    re[r * ld + c] = v.x;
    im[r * ld + c] = v.y;
}

__global__ void interleave_kernel(double* dst, int64_t lwd, const double* re, const double* im, int64_t ld,
                                  int64_t rows, int64_t cols, const int32_t* status) {
    if (status && status[kInfo] != 0) return;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= rows * cols) return;
    const int64_t r = e / cols, c = e - r * cols;
    *reinterpret_cast<double2*>(reinterpret_cast<char*>(dst) + r * lwd + c * 16) =
        make_double2(re[r * ld + c], im[r * ld + c]);
}

// (value, row) with the reference's rule: larger value wins, the lower row among equals; -1 = none
__device__ __forceinline__ void best_of(double& a, int& i, double a2, int i2) {
    if (i2 >= 0 && (i < 0 || a2 > a || (a2 == a && i2 < i))) {
        a = a2;
        i = i2;
    }
}

// Leaf factorisation: rows [0, m), columns [0, w) of the planes (P.re/P.im at the panel's origin).
__global__ void __launch_bounds__(kZPanelThreads) zpanel_kernel(Planes P, int m, int w, int row_base, int col_base,
                                                                int32_t* ipiv, int32_t* status) {
    __shared__ double s_a[kZPanelThreads / 32];
    __shared__ int s_i[kZPanelThreads / 32];
    __shared__ double2 s_u[kZLeaf];  // the pivot row after the interchange
    __shared__ int s_piv, s_stop;
    if (status[kInfo] != 0) return;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    if (t == 0) s_stop = 0;
    for (int j = 0; j < w; ++j) {
        // strict > over rows in ascending order per thread, then the lowest row among equal maxima
        double ba = 0.0;
        int bi = -1;
        for (int i = j + t; i < m; i += kZPanelThreads) {
            const double v = fabs(P.re[(int64_t)i * P.ld + j]) + fabs(P.im[(int64_t)i * P.ld + j]);
            if (v > ba) { ba = v; bi = i; }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double a2 = __shfl_xor_sync(0xffffffffu, ba, o);
            const int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
            best_of(ba, bi, a2, i2);
        }
        if (lane == 0) { s_a[warp] = ba; s_i[warp] = bi; }
        __syncthreads();
        if (warp == 0) {
            ba = s_a[lane];
            bi = s_i[lane];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double a2 = __shfl_xor_sync(0xffffffffu, ba, o);
                const int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
                best_of(ba, bi, a2, i2);
            }
            if (lane == 0) {
                s_piv = bi;
                if (bi < 0 || !(ba > 10.0 / DBL_MAX)) {
                    s_stop = 1;
                    atomicExch(&status[kInfo], 1);
                } else {
                    ipiv[col_base + j] = row_base + bi;
                }
            }
        }
        __syncthreads();
        if (s_stop) return;
        const int p = s_piv;
        // interchange rows j and p over the panel's columns; keep the pivot row for the update
        if (t < w) {
            const int64_t oj = (int64_t)j * P.ld + t, op = (int64_t)p * P.ld + t;
            const double2 vj = make_double2(P.re[oj], P.im[oj]), vp = make_double2(P.re[op], P.im[op]);
            s_u[t] = vp;
            if (p != j) {
                P.re[oj] = vp.x; P.im[oj] = vp.y;
                P.re[op] = vj.x; P.im[op] = vj.y;
            }
        }
        __syncthreads();
        const double2 s = cinv(s_u[j]);
        for (int i = j + 1 + t; i < m; i += kZPanelThreads) {
            const int64_t o = (int64_t)i * P.ld;
            const double2 x = make_double2(P.re[o + j], P.im[o + j]);
            // CAddMul(0, x, s): 0 + x.re s.re - x.im s.im, 0 + x.re s.im + x.im s.re
            const double2 l = make_double2(0.0 + x.x * s.x - x.y * s.y, 0.0 + x.x * s.y + x.y * s.x);
            P.re[o + j] = l.x;
            P.im[o + j] = l.y;
            for (int k = j + 1; k < w; ++k) {
                const double2 a = make_double2(P.re[o + k], P.im[o + k]);
                const double2 r = csub_mul(a, l, s_u[k]);
                P.re[o + k] = r.x;
                P.im[o + k] = r.y;
            }
        }
        __syncthreads();
    }
}

// Triangular solve with the k x k (k <= 32) block T at (tre, tim) (row stride ldt) on ncols columns
// of X (planes, row stride ldx): lower unit (forward) or upper with CDiv (backward).  One warp per
// four columns, lane = row of the block.
constexpr int kZtCpw = 4;
__global__ void __launch_bounds__(128) ztrsm_small_kernel(const double* tre, const double* tim, int64_t ldt,
                                                          double* xre, double* xim, int64_t ldx, int k, int ncols,
                                                          int upper, const int32_t* status) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int c0 = (blockIdx.x * 4 + warp) * kZtCpw;
    if (status[kInfo] != 0 || c0 >= ncols) return;
    double2 trow[kZLeaf];
#pragma unroll
    for (int j = 0; j < kZLeaf; ++j)
        trow[j] = (lane < k && j < k) ? make_double2(tre[(int64_t)lane * ldt + j], tim[(int64_t)lane * ldt + j])
                                      : make_double2(0.0, 0.0);
    double2 x[kZtCpw];
#pragma unroll
    for (int q = 0; q < kZtCpw; ++q)
        x[q] = (lane < k && c0 + q < ncols)
                   ? make_double2(xre[(int64_t)lane * ldx + c0 + q], xim[(int64_t)lane * ldx + c0 + q])
                   : make_double2(0.0, 0.0);
    if (!upper) {
#pragma unroll
        for (int j = 0; j < kZLeaf - 1; ++j) {
            if (j >= k) break;
#pragma unroll
            for (int q = 0; q < kZtCpw; ++q) {
                const double2 xj = make_double2(__shfl_sync(0xffffffffu, x[q].x, j), __shfl_sync(0xffffffffu, x[q].y, j));
                if (lane > j) x[q] = csub_mul(x[q], trow[j], xj);
            }
        }
    } else {
#pragma unroll
        for (int j = kZLeaf - 1; j >= 0; --j) {
            if (j >= k) continue;
#pragma unroll
            for (int q = 0; q < kZtCpw; ++q) {
                if (lane == j) x[q] = cdiv(x[q], trow[j]);
                const double2 xj = make_double2(__shfl_sync(0xffffffffu, x[q].x, j), __shfl_sync(0xffffffffu, x[q].y, j));
                if (lane < j) x[q] = csub_mul(x[q], trow[j], xj);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < kZtCpw; ++q)
        if (lane < k && c0 + q < ncols) {
            xre[(int64_t)lane * ldx + c0 + q] = x[q].x;
            xim[(int64_t)lane * ldx + c0 + q] = x[q].y;
        }
}

// X[i][:] = B[perm[i]][:] on both planes
__global__ void zgather_rows_kernel(double* xre, double* xim, int64_t ldx, const double* bre, const double* bim,
                                    int64_t ldb, const int32_t* perm, int64_t n, int64_t nrhs) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * nrhs) return;
    const int64_t i = e / nrhs, c = e - i * nrhs;
    xre[i * ldx + c] = bre[(int64_t)perm[i] * ldb + c];
    xim[i * ldx + c] = bim[(int64_t)perm[i] * ldb + c];
}

// det = (+-1, 0) * U[0][0] * U[1][1] * ... in order (CMul), 1024 threads
__global__ void __launch_bounds__(1024) zdeterminant_kernel(Planes P, int n, const int32_t* ipiv,
                                                            const int32_t* status, double* det) {
    __shared__ double2 dg[1024];
    __shared__ int flips;
    if (threadIdx.x == 0) flips = 0;
    __syncthreads();
    int local = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (ipiv[i] != i) local++;
    atomicAdd(&flips, local);
    __syncthreads();
    double2 r = make_double2((flips & 1) ? -1.0 : 1.0, 0.0);
    for (int c0 = 0; c0 < n; c0 += 1024) {
        const int i = c0 + (int)threadIdx.x;
        if (i < n) dg[threadIdx.x] = make_double2(P.re[(int64_t)i * P.ld + i], P.im[(int64_t)i * P.ld + i]);
        __syncthreads();
        if (threadIdx.x == 0) {
            const int cnt = min(1024, n - c0);
            for (int k = 0; k < cnt; ++k) {
                const double2 b = dg[k];
                r = make_double2(r.x * b.x - r.y * b.y, r.x * b.y + r.y * b.x);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const bool sing = status[kInfo] != 0;
        det[0] = sing ? 0.0 : r.x;
        det[1] = sing ? 0.0 : r.y;
    }
}

unsigned zblocks(int64_t e) { return (unsigned)ceil_div(std::max<int64_t>(e, 1), 256); }

__global__ void ziota_kernel(int32_t* v, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = (int32_t)i;
}

// C (M x N at c0 of both planes) -= A (M x K) B (K x N) as four real DMMA GEMMs
int32_t zgemm_sub(Ctx* ctx, cudaStream_t st, const Planes& Ap, int64_t an, int64_t ar0, int64_t ac0, const Planes& Bp,
                  int64_t bn, int64_t bcols, int64_t br0, int64_t bc0, const Planes& Cp, int64_t cr0, int64_t cc0,
                  int64_t M, int64_t N, int64_t K) {
    if (M <= 0 || N <= 0 || K <= 0) return B2M_OK;
    DOperand are{Ap.re, Ap.ld, an, an, ar0, ac0, true}, aim{Ap.im, Ap.ld, an, an, ar0, ac0, true};
    DOperand bre{Bp.re, Bp.ld, bn, bcols, br0, bc0, false}, bim{Bp.im, Bp.ld, bn, bcols, br0, bc0, false};
    double* cre = Cp.re + cr0 * Cp.ld + cc0;
    double* cim = Cp.im + cr0 * Cp.ld + cc0;
    B2M_TRY(dgemm_tiled(ctx, st, are, bre, cre, Cp.ld, M, N, K, B2M_DO_SUB, true));
    B2M_TRY(dgemm_tiled(ctx, st, aim, bim, cre, Cp.ld, M, N, K, B2M_DO_ADD, true));
    B2M_TRY(dgemm_tiled(ctx, st, are, bim, cim, Cp.ld, M, N, K, B2M_DO_SUB, true));
    return dgemm_tiled(ctx, st, aim, bre, cim, Cp.ld, M, N, K, B2M_DO_SUB, true);
}

int32_t launch_ztrsm_small(Ctx* ctx, cudaStream_t st, const Planes& T, int64_t r0, const Planes& X, int64_t xr0,
                           int64_t xc0, int k, int ncols, bool upper) {
    if (k <= 0 || ncols <= 0) return B2M_OK;
    ztrsm_small_kernel<<<(unsigned)ceil_div(ncols, 4 * kZtCpw), 128, 0, st>>>(
        T.re + r0 * T.ld + r0, T.im + r0 * T.ld + r0, T.ld, X.re + xr0 * X.ld + xc0, X.im + xr0 * X.ld + xc0, X.ld, k,
        ncols, upper ? 1 : 0, ctx->d_status);
    B2M_LAUNCHED(ctx);
    return B2M_OK;
}

int64_t zsplit(int64_t w) { return round_up((w + 1) / 2, kZLeaf); }

// rows [br0, br0 + k) of X's columns [xc0, xc0 + ncols) <- T(r0..r0+k)^-1 X, T unit lower or upper
int32_t ztrsm_rec(Ctx* ctx, cudaStream_t st, const Planes& T, int64_t tn, int64_t r0, const Planes& X, int64_t xn,
                  int64_t xcols, int64_t br0, int64_t xc0, int64_t ncols, int64_t k, bool upper) {
    if (k <= kZLeaf) return launch_ztrsm_small(ctx, st, T, r0, X, br0, xc0, (int)k, (int)ncols, upper);
    const int64_t k1 = zsplit(k), k2 = k - k1;
    if (!upper) {
        B2M_TRY(ztrsm_rec(ctx, st, T, tn, r0, X, xn, xcols, br0, xc0, ncols, k1, false));
        B2M_TRY(zgemm_sub(ctx, st, T, tn, r0 + k1, r0, X, xn, xcols, br0, xc0, X, br0 + k1, xc0, k2, ncols, k1));
        return ztrsm_rec(ctx, st, T, tn, r0 + k1, X, xn, xcols, br0 + k1, xc0, ncols, k2, false);
    }
    B2M_TRY(ztrsm_rec(ctx, st, T, tn, r0 + k1, X, xn, xcols, br0 + k1, xc0, ncols, k2, true));
    B2M_TRY(zgemm_sub(ctx, st, T, tn, r0, r0 + k1, X, xn, xcols, br0 + k1, xc0, X, br0, xc0, k1, ncols, k2));
    return ztrsm_rec(ctx, st, T, tn, r0, X, xn, xcols, br0, xc0, ncols, k1, true);
}

// factor columns [c0, c0 + width), rows [c0, n)
int32_t zlu_rec(Ctx* ctx, cudaStream_t st, const Planes& A, int64_t n, int64_t c0, int64_t width, int32_t* ipiv,
                int32_t* perm) {
    if (width <= kZLeaf) {
        Planes p{A.re + c0 * A.ld + c0, A.im + c0 * A.ld + c0, A.ld};
        prof_begin(ctx, st, kClsPanel);
        zpanel_kernel<<<1, kZPanelThreads, 0, st>>>(p, (int)(n - c0), (int)width, (int)c0, (int)c0, ipiv,
                                                    ctx->d_status);
        prof_end(ctx, st, kClsPanel, 2.0 * 16.0 * (n - c0) * width);
        B2M_LAUNCHED(ctx);
        B2M_TRY(launch_swaps<double>(ctx, st, A.re, A.ld, (int)n, (int)c0, (int)width, ipiv, perm));
        return launch_swaps<double>(ctx, st, A.im, A.ld, (int)n, (int)c0, (int)width, ipiv, nullptr);
    }
    const int64_t nleft = zsplit(width), nright = width - nleft, r1 = c0 + nleft;
    B2M_TRY(zlu_rec(ctx, st, A, n, c0, nleft, ipiv, perm));
    B2M_TRY(ztrsm_rec(ctx, st, A, n, c0, A, n, n, c0, r1, nright, nleft, false));  // A12 <- L11^-1 A12
    B2M_TRY(zgemm_sub(ctx, st, A, n, r1, c0, A, n, n, c0, r1, A, r1, r1, n - r1, nright, nleft));
    return zlu_rec(ctx, st, A, n, r1, nright, ipiv, perm);
}

}  // namespace

int32_t zlu_factor(Ctx* ctx, cudaStream_t st, double* re, double* im, int64_t ld, int64_t n, int32_t* ipiv,
                   int32_t* perm) {
    if (n <= 0) return B2M_OK;
    if ((ld & 1) || !aligned16(re) || !aligned16(im)) return fail(ctx, B2M_ERR_DIM, "zlu_factor: alignment");
    if (n > (1 << 30)) return fail(ctx, B2M_ERR_UNSUPPORTED, "zlu_factor: n too large");
    const Planes A{re, im, ld};
    const GraphKey key{30, re, im, ipiv, perm, ld, n, 0, 0};
    return run_graph(ctx, st, key, [&](cudaStream_t s) -> int32_t {
        if (perm) {
            ziota_kernel<<<zblocks(n), 256, 0, s>>>(perm, n);
            B2M_LAUNCHED(ctx);
        }
        return zlu_rec(ctx, s, A, n, 0, n, ipiv, perm);
    });
}

int32_t zlu_solve(Ctx* ctx, cudaStream_t st, const double* lre, const double* lim, int64_t ld, int64_t n,
                  const int32_t* perm, double* bre, double* bim, int64_t ldb, int64_t nrhs, double* tre, double* tim) {
    if (n <= 0 || nrhs <= 0) return B2M_OK;
    const Planes L{const_cast<double*>(lre), const_cast<double*>(lim), ld};
    const Planes X{bre, bim, ldb};
    B2M_CU(ctx, cudaMemcpy2DAsync(tre, ldb * 8, bre, ldb * 8, nrhs * 8, n, cudaMemcpyDeviceToDevice, st));
    B2M_CU(ctx, cudaMemcpy2DAsync(tim, ldb * 8, bim, ldb * 8, nrhs * 8, n, cudaMemcpyDeviceToDevice, st));
    zgather_rows_kernel<<<zblocks(n * nrhs), 256, 0, st>>>(bre, bim, ldb, tre, tim, ldb, perm, n, nrhs);
    B2M_LAUNCHED(ctx);
    B2M_TRY(ztrsm_rec(ctx, st, L, n, 0, X, n, nrhs, 0, 0, nrhs, n, false));
    return ztrsm_rec(ctx, st, L, n, 0, X, n, nrhs, 0, 0, nrhs, n, true);
}

int32_t z_deinterleave(Ctx* ctx, cudaStream_t st, const double* src, int64_t lws, double* re, double* im, int64_t ld,
                       int64_t rows, int64_t cols) {
    if (rows <= 0 || cols <= 0) return B2M_OK;
    deinterleave_kernel<<<zblocks(rows * cols), 256, 0, st>>>(src, lws, re, im, ld, rows, cols);
    B2M_LAUNCHED(ctx);
    return B2M_OK;
}

int32_t z_interleave(Ctx* ctx, cudaStream_t st, double* dst, int64_t lwd, const double* re, const double* im,
                     int64_t ld, int64_t rows, int64_t cols, bool only_if_ok) {
    if (rows <= 0 || cols <= 0) return B2M_OK;
    interleave_kernel<<<zblocks(rows * cols), 256, 0, st>>>(dst, lwd, re, im, ld, rows, cols,
                                                            only_if_ok ? ctx->d_status : nullptr);
    B2M_LAUNCHED(ctx);
    return B2M_OK;
}

int32_t z_determinant(Ctx* ctx, cudaStream_t st, const double* re, const double* im, int64_t ld, int64_t n,
                      const int32_t* ipiv, double* d_det2) {
    zdeterminant_kernel<<<1, 1024, 0, st>>>(Planes{const_cast<double*>(re), const_cast<double*>(im), ld}, (int)n,
                                            ipiv, ctx->d_status, d_det2);
    B2M_LAUNCHED(ctx);
    return B2M_OK;
}

}  // namespace b2m
