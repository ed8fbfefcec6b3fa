// lu_mixed.cu -- mixed-precision LU solve: an FP32 factorisation whose trailing updates run on the
// tcgen05 tensor cores (TF32 or 3xTF32, lu_f32.cu), FP64 iterative refinement (residual b - Ax,
// update x += d, normwise backward-error stopping test, all in FP64), and a plain FP64
// re-factorisation when refinement stalls or the FP32 factorisation meets a tiny pivot.
//
// There is no counterpart in the reference (MatrixLinEQSolve, LinAlgLU.pas:481-592, refines a
// fixed number of times in FP64 around an FP64 factorisation); the result is judged against the
// FP64 oracle through its backward error.
//
// One refinement step is a handful of launches, captured once and replayed:
//   * trsv_sweep_kernel, one persistent cooperative launch per triangular sweep (forward with L,
//     backward with U): a CTA per (128-row block, 8 right-hand sides) folds in the earlier blocks
//     as they are published and multiplies by the precomputed inverse and coupling blocks; the
//     backward sweep also adds d to the FP64 solution.  trsv_block_kernel (one launch per block)
//     replaces it when the sweep's CTAs cannot all be resident;
//   * resid_kernel: r = b - A x in FP64 on DMMA (64 rows x 16 right-hand sides per CTA), which also
//     writes P r in FP32 for the next step and the column maxima of |r|, |x| and |b| for the test
//     eta = max_c ||r_c||inf / (||A||inf ||x_c||inf + ||b_c||inf).
#include <cmath>
#include <vector>

#include <cooperative_groups.h>

#include "common.cuh"
#include "kernels.cuh"

namespace cg = cooperative_groups;

namespace b2m {
namespace {

constexpr int kTrRhs = 4;      // right-hand sides per diagonal CTA
constexpr int kTrRows = 64;    // rows per update CTA
constexpr int kTrMaxRhs = 16;  // right-hand sides per sweep launch
constexpr int kReRows = 64;    // rows per residual CTA
constexpr int kReRhs = 16;     // right-hand sides per residual CTA
constexpr int kReK = 64;       // K chunk of the residual
constexpr int kReSplit = 2;    // K halves inside a residual CTA (four warps each)
constexpr int kReStages = 5;   // cp.async pipeline depth (four 44 KiB stages in flight per SM)
constexpr int kReAS = kReK + 2;                                   // A tile row stride (doubles)
constexpr int kReXS = kReRhs + 4;                                 // X tile row stride (doubles)
constexpr int kReStage = kReRows * kReAS + kReK * kReXS;          // doubles per stage
constexpr int kReSmem = kReStages * kReStage * (int)sizeof(double);

unsigned gsz(int64_t n, int b = 256) { return (unsigned)ceil_div(std::max<int64_t>(n, 1), b); }

__device__ __forceinline__ void atomic_max_abs(unsigned long long* p, double v) {
    atomicMax(p, (unsigned long long)__double_as_longlong(fabs(v)));
}

// ||A||inf: max row sum of |a_ij| (one warp per row, then a global max on the bit pattern)
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
    atomic_max_abs(&out[c], R[i * ldr + c]);
    atomic_max_abs(&out[k + c], X[i * ldx + c]);
    atomic_max_abs(&out[2 * k + c], B[i * ldb + c]);
}

// column-wise max |r| of R (n x k) into out[0..k) (bit patterns)
__global__ void colmax_kernel(const double* R, int64_t ldr, int64_t n, int64_t k, unsigned long long* out) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * k) return;
    const int64_t i = e / k, c = e - i * k;
    atomic_max_abs(&out[c], R[i * ldr + c]);
}

// FP32 copy of A and ||A||inf in one pass over A: a warp per row (grid-stride over rows), each lane
// converting and summing |a_ij| over its columns j = lane, lane + 32, ... in order (the same sum as
// norm_inf_kernel), four loads in flight; the row sums meet in a global max on the bit pattern.
__global__ void __launch_bounds__(256) f64_to_f32_norm_kernel(const double* src, int64_t lds, float* dst, int64_t ldd,
                                                              int64_t n, unsigned long long* out) {
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x / 32);
    for (int64_t row = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); row < n; row += nwarps) {
        const double* a = src + row * lds;
        float* d = dst + row * ldd;
        double s = 0.0;
        int64_t j = lane;
        for (; j + 96 < n; j += 128) {
            const double v0 = a[j], v1 = a[j + 32], v2 = a[j + 64], v3 = a[j + 96];
            d[j] = (float)v0; d[j + 32] = (float)v1; d[j + 64] = (float)v2; d[j + 96] = (float)v3;
            s += fabs(v0); s += fabs(v1); s += fabs(v2); s += fabs(v3);
        }
        for (; j < n; j += 32) {
            const double v = a[j];
            d[j] = (float)v;
            s += fabs(v);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) atomicMax(out, (unsigned long long)__double_as_longlong(s));
    }
}

// pinv[perm[i]] = i
__global__ void invert_perm_kernel(const int32_t* perm, int32_t* pinv, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) pinv[perm[i]] = (int32_t)i;
}

// start of refinement: x = 0, r32 = P b
__global__ void ir_init_kernel(const double* B, int64_t ldb, const int32_t* perm, float* r32, int64_t ldr, double* X,
                               int64_t ldx, int64_t n, int64_t nrhs) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * nrhs) return;
    const int64_t i = e / nrhs, c = e - i * nrhs;
    r32[i * ldr + c] = (float)B[(int64_t)perm[i] * ldb + c];
    X[i * ldx + c] = 0.0;
}

struct TrArgs {
    const float* T;     // the FP32 factors (unit-lower L below the diagonal, U on and above)
    int64_t ld;
    int n;
    const float* inv;   // inverses of the diagonal blocks, kTrsvNB x kTrsvNB each
    float* Xr;          // right-hand sides / solution (n x ldr), columns [c0, c0 + nc)
    int64_t ldr;
    int c0, nc;
    double* X64;        // backward sweep: X64 += solution
    int64_t ldx;
    int upper;
    int nd;             // diagonal CTAs
    const int32_t* status;
};

// One block step of a blocked triangular solve.  Block b's diagonal CTAs (kTrRhs columns each)
// subtract block `prev`'s contribution from block b and multiply by inv(T_bb); the update CTAs
// subtract block `prev`'s contribution from the rows still to come (below b when forward, above b
// when backward).  Rows of T are read as float4 straight into registers (a row of the factors
// starts 128-byte aligned), so every thread has all of its loads in flight at once.
__device__ __forceinline__ float4 ld_row4(const float* row, int k, int kmax) {
    if (k >= kmax) return make_float4(0.f, 0.f, 0.f, 0.f);
    float4 v = __ldg(reinterpret_cast<const float4*>(row + k));
    if (k + 1 >= kmax) v.y = 0.f;  // the factors' padding columns are never initialised
    if (k + 2 >= kmax) v.z = 0.f;
    if (k + 3 >= kmax) v.w = 0.f;
    return v;
}

constexpr int kSwTS = kTrsvNB + 4;  // line stride of the staged T_bj (528 bytes: 16-byte aligned lines)

// T_bj (128 x 128) into shared memory, row r at r * kSwTS floats (the stride keeps the fold's float4
// reads of one column group by 32 consecutive rows at four wavefronts, the minimum).  A full block
// comes in as 128 bulk copies of 512 bytes (one instruction per row, the FP32 factors' rows are
// 16-byte aligned: their leading dimension is a multiple of 32) completing on `bar`; a partial one
// by asynchronous 16-byte copies, zero past the matrix and in the factors' padding columns.
__device__ __forceinline__ bool sw_stage(float* s_tt, const float* T, int64_t ld, int b0, int bs, int p0, int ps,
                                         int t, uint64_t* bar) {
    if (bs == kTrsvNB && ps == kTrsvNB) {
        if (t == 0) mbar_arrive_expect_tx(bar, kTrsvNB * kTrsvNB * (int)sizeof(float));
        if (t < kTrsvNB) bulk_g2s(s_tt + t * kSwTS, T + (int64_t)(b0 + t) * ld + p0, kTrsvNB * (int)sizeof(float), bar);
        return true;
    }
#pragma unroll 4
    for (int i = 0; i < kTrsvNB * kTrsvNB / (4 * 256); ++i) {
        const int e = t + 256 * i;
        const int rr = e >> 5, c4 = e & 31;
        const int nb = rr < bs ? 4 * max(0, min(4, ps - 4 * c4)) : 0;
        const float* src = nb > 0 ? T + (int64_t)(b0 + rr) * ld + p0 + 4 * c4 : T;
        cp_async16(s_tt + rr * kSwTS + 4 * c4, src, nb);
    }
    cp_async_commit();
    return false;
}
__device__ __forceinline__ float4 sw_tile4(const float* s_tt, int r, int c4) {
    return *reinterpret_cast<const float4*>(s_tt + r * kSwTS + 4 * c4);
}

__global__ void __launch_bounds__(256) trsv_block_kernel(TrArgs a, int b) {
    __shared__ __align__(16) float s_p[kTrsvNB][kTrMaxRhs];  // solution of block prev
    __shared__ __align__(16) float s_y[kTrsvNB][kTrRhs];
    __shared__ __align__(16) float s_h[kTrsvNB][kTrRhs];     // second-half partial sums
    if (a.status[kInfo] != 0) return;
    const int t = threadIdx.x;
    const int NB = kTrsvNB;
    const int nblk = (int)ceil_div(a.n, NB);
    const int prev = a.upper ? b + 1 : b - 1;
    const bool has_prev = prev >= 0 && prev < nblk;
    const int p0 = prev * NB, ps = has_prev ? min(NB, a.n - p0) : 0;
    const int b0 = b * NB, bs = min(NB, a.n - b0);
    if (blockIdx.x < a.nd) {
        const int g = blockIdx.x * kTrRhs;  // first column of this CTA's group, relative to c0
        const int r = t & (NB - 1), h = t >> 7;  // row r, K half h
        // every global load of this CTA is issued before the first barrier
        float4 tv[16], iv[16];
        {
            const float* trow = a.T + (int64_t)(b0 + min(r, bs - 1)) * a.ld + p0;
            const float* irow = a.inv + (int64_t)b * NB * NB + (int64_t)r * NB + 64 * h;
#pragma unroll
            for (int i = 0; i < 16; ++i) tv[i] = (r < bs && has_prev) ? ld_row4(trow, 64 * h + 4 * i, ps) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
            for (int i = 0; i < 16; ++i) iv[i] = __ldg(reinterpret_cast<const float4*>(irow) + i);
        }
        float xb[kTrRhs];
#pragma unroll
        for (int q = 0; q < kTrRhs; ++q)
            xb[q] = (h == 0 && r < bs && g + q < a.nc) ? a.Xr[(int64_t)(b0 + r) * a.ldr + a.c0 + g + q] : 0.f;
        {
            float v[2];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int e = t + 256 * i, k = e >> 2, q = e & 3;
                v[i] = (k < ps && g + q < a.nc) ? a.Xr[(int64_t)(p0 + k) * a.ldr + a.c0 + g + q] : 0.f;
            }
#pragma unroll
            for (int i = 0; i < 2; ++i) s_p[(t + 256 * i) >> 2][(t + 256 * i) & 3] = v[i];
        }
        __syncthreads();
        // y = X_b - T_{b,prev} X_prev
        float acc[kTrRhs] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const float tk[4] = {tv[i].x, tv[i].y, tv[i].z, tv[i].w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const float4 xp = *reinterpret_cast<const float4*>(&s_p[64 * h + 4 * i + e][0]);
                acc[0] = fmaf(tk[e], xp.x, acc[0]);
                acc[1] = fmaf(tk[e], xp.y, acc[1]);
                acc[2] = fmaf(tk[e], xp.z, acc[2]);
                acc[3] = fmaf(tk[e], xp.w, acc[3]);
            }
        }
        if (h == 1) *reinterpret_cast<float4*>(&s_h[r][0]) = make_float4(acc[0], acc[1], acc[2], acc[3]);
        __syncthreads();
        if (h == 0) {
            const float4 o = *reinterpret_cast<const float4*>(&s_h[r][0]);
            const float oh[4] = {o.x, o.y, o.z, o.w};
#pragma unroll
            for (int q = 0; q < kTrRhs; ++q) s_y[r][q] = (r < bs) ? xb[q] - acc[q] - oh[q] : 0.f;
        }
        __syncthreads();
        // x_b = inv(T_bb) y (the inverse is zero outside the block's extent)
        float x[kTrRhs] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const float ik[4] = {iv[i].x, iv[i].y, iv[i].z, iv[i].w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const float4 y = *reinterpret_cast<const float4*>(&s_y[64 * h + 4 * i + e][0]);
                x[0] = fmaf(ik[e], y.x, x[0]);
                x[1] = fmaf(ik[e], y.y, x[1]);
                x[2] = fmaf(ik[e], y.z, x[2]);
                x[3] = fmaf(ik[e], y.w, x[3]);
            }
        }
        if (h == 1) *reinterpret_cast<float4*>(&s_h[r][0]) = make_float4(x[0], x[1], x[2], x[3]);
        __syncthreads();
        if (h == 0 && r < bs) {
            const float4 o = *reinterpret_cast<const float4*>(&s_h[r][0]);
            const float oh[4] = {o.x, o.y, o.z, o.w};
#pragma unroll
            for (int q = 0; q < kTrRhs; ++q) {
                if (g + q >= a.nc) continue;
                const float v = x[q] + oh[q];
                const int64_t col = a.c0 + g + q;
                a.Xr[(int64_t)(b0 + r) * a.ldr + col] = v;
                if (a.upper) a.X64[(int64_t)(b0 + r) * a.ldx + col] += (double)v;
            }
        }
        return;
    }
    if (!has_prev) return;
    // update CTA: rows [u0, u0 + kTrRows) of the remaining range; 4 lanes per row split K in
    // quarters.  s_p rows are stored with their 16-byte chunks rotated by (k >> 5) so that the four
    // quarter-groups of a warp read different banks.
    const int u = blockIdx.x - a.nd;
    const int u0 = a.upper ? u * kTrRows : b0 + bs + u * kTrRows;
    const int uend = a.upper ? b0 : a.n;
    if (u0 >= uend) return;
    const int rr = t >> 2, kq = t & 3;
    const int row = u0 + rr;
    float4 tv[8];
    {
        const float* trow = a.T + (int64_t)min(row, uend - 1) * a.ld + p0;
#pragma unroll
        for (int i = 0; i < 8; ++i) tv[i] = row < uend ? ld_row4(trow, 32 * kq + 4 * i, ps) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    {
        float v[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int e = t + 256 * i, k = e >> 4, c = e & 15;
            v[i] = (k < ps && c < a.nc) ? a.Xr[(int64_t)(p0 + k) * a.ldr + a.c0 + c] : 0.f;
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int e = t + 256 * i, k = e >> 4, c = e & 15;
            s_p[k][(((c >> 2) ^ (k >> 5)) & 3) * 4 + (c & 3)] = v[i];
        }
    }
    __syncthreads();
    float acc[kTrMaxRhs];
#pragma unroll
    for (int c = 0; c < kTrMaxRhs; ++c) acc[c] = 0.f;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const float tk[4] = {tv[i].x, tv[i].y, tv[i].z, tv[i].w};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int k = 32 * kq + 4 * i + e;
            const float* xp = &s_p[k][0];
#pragma unroll
            for (int c4 = 0; c4 < kTrMaxRhs / 4; ++c4) {
                const float4 xv = *reinterpret_cast<const float4*>(xp + ((c4 ^ kq) & 3) * 4);
                acc[4 * c4 + 0] = fmaf(tk[e], xv.x, acc[4 * c4 + 0]);
                acc[4 * c4 + 1] = fmaf(tk[e], xv.y, acc[4 * c4 + 1]);
                acc[4 * c4 + 2] = fmaf(tk[e], xv.z, acc[4 * c4 + 2]);
                acc[4 * c4 + 3] = fmaf(tk[e], xv.w, acc[4 * c4 + 3]);
            }
        }
    }
#pragma unroll
    for (int c = 0; c < kTrMaxRhs; ++c) {
        acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], 1);
        acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], 2);
    }
    if (row < uend) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int c = 4 * kq + i;
            if (c < a.nc) a.Xr[(int64_t)row * a.ldr + a.c0 + c] -= acc[c];
        }
    }
}


// ------------------------------------------------------------------ persistent sweep
// One cooperative launch per sweep: CTA (block b, group g) owns rows [128 b, +128) and right-hand
// sides [8 g, +8).  With T_bb^-1 and the coupling block W_b = T_bb^-1 T_{b,p} (p the block solved
// just before b) precomputed, the block's solution is
//     x_b = T_bb^-1 (X_b - sum_{j before p} T_bj x_j)  -  W_b x_p,
// so everything but the last product is done while block p is still being solved, and the chain
// of 128-row blocks advances by one 128 x 128 x 8 product and one L2 round trip per step: a block's
// solution is published as 64-bit words {value, flag} (written and polled with single 64-bit
// accesses, so a word whose flag is set carries its value; no fence, no separate flag read).
// T_bb^-1 and W_b are staged in shared memory at kernel start, the rows of the other T_bj are
// loaded into registers before each wait.  All CTAs are resident (cooperative launch); every wait
// is bounded and reports a timeout through the status words, and a CTA that gives up marks its
// words with the flag kSwAbort so that the CTAs after it give up without waiting again.
constexpr int kSwRhs = 8;
constexpr uint32_t kSwSpin = 1u << 22;
constexpr uint32_t kSwAbort = 0xFFFFFFFFu;
constexpr int kSwSmem = (2 * kTrsvNB * kTrsvNB + kTrsvNB * kSwTS) * (int)sizeof(float);  // T_bb^-1, W_b, T_bj

struct SwArgs {
    const float* T;
    int64_t ld;
    int n;
    const float* inv;  // T_bb^-1 per block (128 x 128, zero padded)
    const float* w;    // W_b per block (128 x 128, zero padded; unused for the first block)
    float* Xr;
    int64_t ldr;
    int c0, nc;
    double* X64;
    int64_t ldx;
    int upper;
    unsigned long long* ll;  // [nblk][ng][128][8] published solutions {value bits, flag}, zeroed before the launch
    int32_t* status;
    uint32_t spin;  // polls before a wait gives up (kSwSpin unless a test lowered it)
};

__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];\n" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;\n" ::"l"(p), "l"(v) : "memory");
}

// acc[q] += sum over this thread's 64 k of M[r][k] * P[k][q], M staged as float4 [k/4][row].
__device__ __forceinline__ void sw_smem_product(const float4* sM, int r, int h, const float (*P)[kSwRhs],
                                                float (&acc)[kSwRhs]) {
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const float4 m = sM[(16 * h + i) * kTrsvNB + r];
        const float mk[4] = {m.x, m.y, m.z, m.w};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int k = 64 * h + 4 * i + e;
            const float4 x0 = *reinterpret_cast<const float4*>(&P[k][0]);
            const float4 x1 = *reinterpret_cast<const float4*>(&P[k][4]);
            acc[0] = fmaf(mk[e], x0.x, acc[0]);
            acc[1] = fmaf(mk[e], x0.y, acc[1]);
            acc[2] = fmaf(mk[e], x0.z, acc[2]);
            acc[3] = fmaf(mk[e], x0.w, acc[3]);
            acc[4] = fmaf(mk[e], x1.x, acc[4]);
            acc[5] = fmaf(mk[e], x1.y, acc[5]);
            acc[6] = fmaf(mk[e], x1.z, acc[6]);
            acc[7] = fmaf(mk[e], x1.w, acc[7]);
        }
    }
}

__global__ void __launch_bounds__(256, 1) trsv_sweep_kernel(SwArgs a) {
    extern __shared__ __align__(16) float4 sw_dyn[];
    __shared__ __align__(16) float s_p[kTrsvNB][kSwRhs];  // x of the block being folded in
    __shared__ __align__(16) float s_y[kTrsvNB][kSwRhs];
    __shared__ __align__(16) float s_h[kTrsvNB][kSwRhs];
    __shared__ int s_abort;
    float4* s_inv = sw_dyn;                        // [32][128]: s_inv[kq][r] = inv[r][4kq .. 4kq+3]
    float4* s_w = sw_dyn + kTrsvNB * kTrsvNB / 4;  // same layout for W_b
    float* s_tt = reinterpret_cast<float*>(sw_dyn + kTrsvNB * kTrsvNB / 2);  // T_bj being folded in
    const int t = threadIdx.x;
    if (a.status[kInfo] != 0) return;
    const int NB = kTrsvNB;
    const int nblk = (int)ceil_div(a.n, NB);
    const int ng = (int)ceil_div(a.nc, kSwRhs);
    const int bi = blockIdx.x / ng, g = blockIdx.x - bi * ng;
    const int b = a.upper ? nblk - 1 - bi : bi;
    const int b0 = b * NB, bs = min(NB, a.n - b0);
    const int r = t & (NB - 1), h = t >> 7;
    const int cg = a.c0 + g * kSwRhs;
    const int ncg = min(kSwRhs, a.nc - g * kSwRhs);
    __shared__ __align__(8) uint64_t s_tbar;  // completion of a bulk-staged T_bj
    if (t == 0) {
        s_abort = 0;
        mbar_init(&s_tbar, 1);
        fence_barrier_init();
    }
    __syncthreads();
    uint32_t tphase = 0;
    bool tbulk = false;  // a bulk copy of T_bj is in flight (uniform)
    {
        const float* inv = a.inv + (int64_t)b * NB * NB;
        const float* w = a.w + (int64_t)b * NB * NB;
#pragma unroll 4
        for (int i = 0; i < 16; ++i) {
            const int e = t + 256 * i, rr = e & (NB - 1), kq = e >> 7;
            cp_async16(s_inv + kq * NB + rr, inv + rr * NB + 4 * kq, 16);
            if (bi > 0) cp_async16(s_w + kq * NB + rr, w + rr * NB + 4 * kq, 16);
        }
        cp_async_commit();
    }
    float xb[kSwRhs];  // own right-hand side (h == 0 threads)
#pragma unroll
    for (int q = 0; q < kSwRhs; ++q)
        xb[q] = (h == 0 && r < bs && q < ncg) ? a.Xr[(int64_t)(b0 + r) * a.ldr + cg + q] : 0.f;
    float acc[kSwRhs];
#pragma unroll
    for (int q = 0; q < kSwRhs; ++q) acc[q] = 0.f;

    // this CTA's published words; thread t polls rows t / 2, columns 4 (t % 2) .. + 3 of a block
    unsigned long long* ll_own = a.ll + (size_t)(b * ng + g) * (kTrsvNB * kSwRhs);
    auto abandon = [&]() {  // mark every word of this CTA so that its dependants stop at once
#pragma unroll
        for (int e = 0; e < 4; ++e) st_relaxed64(ll_own + 4 * t + e, (unsigned long long)kSwAbort << 32);
    };
    // wait for block j of the sweep and stage its solution in s_p; false if the sweep is abandoned
    auto wait_and_stage = [&](int j) -> bool {
        const int k = t >> 1, q0 = (t & 1) * 4;
        const unsigned long long* src = a.ll + (size_t)(j * ng + g) * (kTrsvNB * kSwRhs) + k * kSwRhs + q0;
        unsigned long long w[4] = {0ull, 0ull, 0ull, 0ull};
        bool ready = false, bad = false;
        for (uint32_t it = 0; it < a.spin && !ready && !bad; ++it) {
#pragma unroll
            for (int e = 0; e < 4; ++e) w[e] = ld_relaxed64(src + e);
            ready = true;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const uint32_t f = (uint32_t)(w[e] >> 32);
                ready = ready && f == 1u;
                bad = bad || f == kSwAbort;
            }
        }
        if (!ready && !bad) atomicExch(&a.status[kTimeout], 501);
        if (!ready) s_abort = 1;
        const float4 v = make_float4(__uint_as_float((uint32_t)w[0]), __uint_as_float((uint32_t)w[1]),
                                     __uint_as_float((uint32_t)w[2]), __uint_as_float((uint32_t)w[3]));
        *reinterpret_cast<float4*>(&s_p[k][q0]) = v;
        cp_async_wait<0>();  // this thread's part of T_bj has landed
        if (tbulk) {  // so have the bulk copies (waited for even when the block wait gave up)
            if (!mbar_wait(&s_tbar, tphase, &a.status[kTimeout], 507)) s_abort = 1;
            tphase ^= 1u;
            tbulk = false;
        }
        __syncthreads();
        if (s_abort) {
            abandon();
            return false;
        }
        return true;
    };

    // all blocks before the last one: contributions with T_bj staged in shared memory
    for (int jj = 0; jj + 1 < bi; ++jj) {
        const int j = a.upper ? nblk - 1 - jj : jj;
        const int p0 = j * NB, ps = min(NB, a.n - p0);
        tbulk = sw_stage(s_tt, a.T, a.ld, b0, bs, p0, ps, t, &s_tbar);  // in flight during the wait
        if (!wait_and_stage(j)) return;
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const float4 tvi = sw_tile4(s_tt, r, 16 * h + i);
            const float tk[4] = {tvi.x, tvi.y, tvi.z, tvi.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int k = 64 * h + 4 * i + e;
                const float4 x0 = *reinterpret_cast<const float4*>(&s_p[k][0]);
                const float4 x1 = *reinterpret_cast<const float4*>(&s_p[k][4]);
                acc[0] = fmaf(tk[e], x0.x, acc[0]);
                acc[1] = fmaf(tk[e], x0.y, acc[1]);
                acc[2] = fmaf(tk[e], x0.z, acc[2]);
                acc[3] = fmaf(tk[e], x0.w, acc[3]);
                acc[4] = fmaf(tk[e], x1.x, acc[4]);
                acc[5] = fmaf(tk[e], x1.y, acc[5]);
                acc[6] = fmaf(tk[e], x1.z, acc[6]);
                acc[7] = fmaf(tk[e], x1.w, acc[7]);
            }
        }
        __syncthreads();  // s_p is rewritten by the next block
    }
    // y = X_b - sum_{j before p} T_bj x_j ;  z = T_bb^-1 y
    if (h == 1) {
#pragma unroll
        for (int q = 0; q < kSwRhs; ++q) s_h[r][q] = acc[q];
    }
    cp_async_wait<0>();
    __syncthreads();
    if (h == 0) {
#pragma unroll
        for (int q = 0; q < kSwRhs; ++q) s_y[r][q] = xb[q] - acc[q] - s_h[r][q];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kSwRhs; ++q) acc[q] = 0.f;
    sw_smem_product(s_inv, r, h, s_y, acc);
    if (bi > 0) {  // x_b = z - W_b x_p
        const int p = a.upper ? b + 1 : b - 1;
        if (!wait_and_stage(p)) return;
#pragma unroll
        for (int q = 0; q < kSwRhs; ++q) acc[q] = -acc[q];
        sw_smem_product(s_w, r, h, s_p, acc);
#pragma unroll
        for (int q = 0; q < kSwRhs; ++q) acc[q] = -acc[q];
    }
    if (h == 1) {
#pragma unroll
        for (int q = 0; q < kSwRhs; ++q) s_h[r][q] = acc[q];
    }
    __syncthreads();
    float xv[kSwRhs];
    if (h == 0) {  // publish every word of the block (zeros past the matrix and past the right-hand sides)
#pragma unroll
        for (int q = 0; q < kSwRhs; ++q) {
            xv[q] = (r < bs && q < ncg) ? acc[q] + s_h[r][q] : 0.f;
            st_relaxed64(ll_own + r * kSwRhs + q, (1ull << 32) | __float_as_uint(xv[q]));
        }
        if (r < bs) {
#pragma unroll
            for (int q = 0; q < kSwRhs; ++q)
                if (q < ncg) a.Xr[(int64_t)(b0 + r) * a.ldr + cg + q] = xv[q];
        }
    }
    if (a.upper && h == 0 && r < bs) {  // the FP64 accumulation is off the chain
#pragma unroll
        for (int q = 0; q < kSwRhs; ++q)
            if (q < ncg) a.X64[(int64_t)(b0 + r) * a.ldx + cg + q] += (double)xv[q];
    }
}

// Chained variant of trsv_sweep_kernel on thread-block clusters of kChCl (8 or 4) consecutive blocks (in
// sweep order, one right-hand-side group per cluster row): besides publishing its solution to
// global memory, a block pushes it into the shared memory of every later block of its cluster
// (st.async completing on the receiver's mbarrier for that sender, 4 KiB each), and a block folds
// the earlier blocks of its own cluster in from there.  Only the hop into the first block of a
// cluster pays a round trip through L2; the others ride on distributed shared memory.  Every
// wait is bounded; a wait that gives up flags status[kTimeout], which every other wait also polls,
// so the whole sweep winds down quickly.  All CTAs of a cluster meet at a cluster barrier after
// the mbarriers are initialised and before they exit.
constexpr int kChSlot = kTrsvNB * kSwRhs * (int)sizeof(float);        // one pushed solution block
template <int CL>
constexpr int chain_smem() { return kSwSmem + (CL - 1) * kChSlot; }  // + receive slots

__device__ __forceinline__ int ld_volatile_i32(const int32_t* p) { return *reinterpret_cast<const volatile int32_t*>(p); }

template <int kChCl>
__global__ void __cluster_dims__(kChCl, 1, 1) __launch_bounds__(256, 1) trsv_chain_kernel(SwArgs a, int nbp) {
    extern __shared__ __align__(16) float4 sw_dyn[];
    __shared__ __align__(16) float s_p[kTrsvNB][kSwRhs];  // x of a block from another cluster
    __shared__ __align__(16) float s_y[kTrsvNB][kSwRhs];
    __shared__ __align__(16) float s_h[kTrsvNB][kSwRhs];
    __shared__ __align__(8) uint64_t s_bar[kChCl];       // one per earlier block of the cluster
    __shared__ int s_abort;
    float4* s_inv = sw_dyn;                        // [32][128]: s_inv[kq][r] = inv[r][4kq .. 4kq+3]
    float4* s_w = sw_dyn + kTrsvNB * kTrsvNB / 4;  // same layout for W_b
    float* s_tt = reinterpret_cast<float*>(sw_dyn + kTrsvNB * kTrsvNB / 2);  // T_bj being folded in
    float (*s_rx)[kTrsvNB][kSwRhs] =
        reinterpret_cast<float (*)[kTrsvNB][kSwRhs]>(sw_dyn + kTrsvNB * kTrsvNB / 2 + kTrsvNB * kSwTS / 4);
    if (a.status[kInfo] != 0) return;  // uniform: written before the launch
    cg::cluster_group cluster = cg::this_cluster();
    const int t = threadIdx.x;
    const int NB = kTrsvNB;
    const int nblk = (int)ceil_div(a.n, NB);
    const int g = blockIdx.x / nbp, bi = blockIdx.x - g * nbp;
    const int rank = (int)cluster.block_rank();  // bi % kChCl: nbp is a multiple of kChCl
    const int cl0 = bi - rank;
    __shared__ __align__(8) uint64_t s_tbar;  // completion of a bulk-staged T_bj
    if (t == 0) {
        for (int q = 0; q < rank; ++q) mbar_init(&s_bar[q], 1);
        mbar_init(&s_tbar, 1);
        fence_barrier_init();
        for (int q = 0; q < rank; ++q) mbar_arrive_expect_tx(&s_bar[q], kChSlot);
        s_abort = 0;
    }
    uint32_t tphase = 0;
    bool tbulk = false;  // a bulk copy of T_bj is in flight (uniform)
    cluster.sync();  // every receiver's mbarriers are armed before the first push
    if (bi >= nblk) {  // padding CTA of the last cluster
        cluster.sync();
        return;
    }
    const int b = a.upper ? nblk - 1 - bi : bi;
    const int b0 = b * NB, bs = min(NB, a.n - b0);
    const int r = t & (NB - 1), h = t >> 7;
    const int cgc = a.c0 + g * kSwRhs;
    const int ncg = min(kSwRhs, a.nc - g * kSwRhs);
    {
        const float* inv = a.inv + (int64_t)b * NB * NB;
        const float* w = a.w + (int64_t)b * NB * NB;
#pragma unroll 4
        for (int i = 0; i < 16; ++i) {
            const int e = t + 256 * i, rr = e & (NB - 1), kq = e >> 7;
            cp_async16(s_inv + kq * NB + rr, inv + rr * NB + 4 * kq, 16);
            if (bi > 0) cp_async16(s_w + kq * NB + rr, w + rr * NB + 4 * kq, 16);
        }
        cp_async_commit();
    }
    float xb[kSwRhs];
#pragma unroll
    for (int q = 0; q < kSwRhs; ++q)
        xb[q] = (h == 0 && r < bs && q < ncg) ? a.Xr[(int64_t)(b0 + r) * a.ldr + cgc + q] : 0.f;
    float acc[kSwRhs];
#pragma unroll
    for (int q = 0; q < kSwRhs; ++q) acc[q] = 0.f;
    const int ng = (int)ceil_div(a.nc, kSwRhs);
    unsigned long long* ll_own = a.ll + (size_t)(b * ng + g) * (kTrsvNB * kSwRhs);
    int32_t* tmo = &a.status[kTimeout];
    auto abandon = [&]() {
#pragma unroll
        for (int e = 0; e < 4; ++e) st_relaxed64(ll_own + 4 * t + e, (unsigned long long)kSwAbort << 32);
    };
    // block j (sweep position jj) from another cluster: global words into s_p
    auto wait_global = [&](int j) -> bool {
        const int k = t >> 1, q0 = (t & 1) * 4;
        const unsigned long long* src = a.ll + (size_t)(j * ng + g) * (kTrsvNB * kSwRhs) + k * kSwRhs + q0;
        unsigned long long w[4] = {0ull, 0ull, 0ull, 0ull};
        bool ready = false, bad = false;
        for (uint32_t it = 0; it < a.spin && !ready && !bad; ++it) {
#pragma unroll
            for (int e = 0; e < 4; ++e) w[e] = ld_relaxed64(src + e);
            ready = true;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const uint32_t f = (uint32_t)(w[e] >> 32);
                ready = ready && f == 1u;
                bad = bad || f == kSwAbort;
            }
            if ((it & 255u) == 255u && ld_volatile_i32(tmo) != 0) bad = true;
        }
        if (!ready && !bad) atomicCAS(tmo, 0, 503);
        if (!ready) s_abort = 1;
        const float4 v = make_float4(__uint_as_float((uint32_t)w[0]), __uint_as_float((uint32_t)w[1]),
                                     __uint_as_float((uint32_t)w[2]), __uint_as_float((uint32_t)w[3]));
        *reinterpret_cast<float4*>(&s_p[k][q0]) = v;
        cp_async_wait<0>();  // this thread's part of T_bj has landed
        if (tbulk) {  // so have the bulk copies (waited for even when the block wait gave up)
            if (!mbar_wait(&s_tbar, tphase, &a.status[kTimeout], 508)) s_abort = 1;
            tphase ^= 1u;
            tbulk = false;
        }
        __syncthreads();
        return !s_abort;
    };
    // the push of cluster rank q into s_rx[q]
    auto wait_push = [&](int q) -> bool {
        bool ready = false, bad = false;
        for (uint32_t it = 0; it < a.spin && !ready && !bad; ++it) {
            ready = mbar_try_wait_cluster(&s_bar[q], 0);
            if (!ready && (it & 255u) == 255u && ld_volatile_i32(tmo) != 0) bad = true;
        }
        if (!ready && !bad) atomicCAS(tmo, 0, 504);
        if (!ready) s_abort = 1;
        cp_async_wait<0>();  // this thread's part of T_bj has landed
        if (tbulk) {  // so have the bulk copies (waited for even when the block wait gave up)
            if (!mbar_wait(&s_tbar, tphase, &a.status[kTimeout], 509)) s_abort = 1;
            tphase ^= 1u;
            tbulk = false;
        }
        __syncthreads();
        return !s_abort;
    };

    bool ok = true;
    for (int jj = 0; ok && jj + 1 < bi; ++jj) {
        const int j = a.upper ? nblk - 1 - jj : jj;
        const int p0 = j * NB, ps = min(NB, a.n - p0);
        tbulk = sw_stage(s_tt, a.T, a.ld, b0, bs, p0, ps, t, &s_tbar);  // in flight during the wait
        const bool local = jj >= cl0;
        ok = local ? wait_push(jj - cl0) : wait_global(j);
        if (!ok) break;
        const float (*P)[kSwRhs] = local ? s_rx[jj - cl0] : s_p;
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const float4 tvi = sw_tile4(s_tt, r, 16 * h + i);
            const float tk[4] = {tvi.x, tvi.y, tvi.z, tvi.w};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int k = 64 * h + 4 * i + e;
                const float4 x0 = *reinterpret_cast<const float4*>(&P[k][0]);
                const float4 x1 = *reinterpret_cast<const float4*>(&P[k][4]);
                acc[0] = fmaf(tk[e], x0.x, acc[0]);
                acc[1] = fmaf(tk[e], x0.y, acc[1]);
                acc[2] = fmaf(tk[e], x0.z, acc[2]);
                acc[3] = fmaf(tk[e], x0.w, acc[3]);
                acc[4] = fmaf(tk[e], x1.x, acc[4]);
                acc[5] = fmaf(tk[e], x1.y, acc[5]);
                acc[6] = fmaf(tk[e], x1.z, acc[6]);
                acc[7] = fmaf(tk[e], x1.w, acc[7]);
            }
        }
        __syncthreads();  // s_p is rewritten by the next global wait
    }
    if (ok) {
        if (h == 1) {
#pragma unroll
            for (int q = 0; q < kSwRhs; ++q) s_h[r][q] = acc[q];
        }
        cp_async_wait<0>();
        __syncthreads();
        if (h == 0) {
#pragma unroll
            for (int q = 0; q < kSwRhs; ++q) s_y[r][q] = xb[q] - acc[q] - s_h[r][q];
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < kSwRhs; ++q) acc[q] = 0.f;
        sw_smem_product(s_inv, r, h, s_y, acc);
        if (bi > 0) {  // x_b = z - W_b x_p
            const bool local = bi - 1 >= cl0;
            ok = local ? wait_push(bi - 1 - cl0) : wait_global(a.upper ? b + 1 : b - 1);
            if (ok) {
#pragma unroll
                for (int q = 0; q < kSwRhs; ++q) acc[q] = -acc[q];
                sw_smem_product(s_w, r, h, local ? s_rx[bi - 1 - cl0] : s_p, acc);
#pragma unroll
                for (int q = 0; q < kSwRhs; ++q) acc[q] = -acc[q];
            }
        }
    }
    if (ok) {
        if (h == 1) {
#pragma unroll
            for (int q = 0; q < kSwRhs; ++q) s_h[r][q] = acc[q];
        }
        __syncthreads();
        if (h == 0) {
            float xv[kSwRhs];
#pragma unroll
            for (int q = 0; q < kSwRhs; ++q) xv[q] = (r < bs && q < ncg) ? acc[q] + s_h[r][q] : 0.f;
            // the later blocks of this cluster first (they are on the chain), then global memory
            for (int d = rank + 1; d < kChCl && cl0 + d < nblk; ++d) {
                const uint32_t rb = map_rank(&s_bar[rank], (uint32_t)d);
                const uint32_t dst = map_rank(&s_rx[rank][r][0], (uint32_t)d);
                st_async16(dst, make_uint4(__float_as_uint(xv[0]), __float_as_uint(xv[1]), __float_as_uint(xv[2]),
                                           __float_as_uint(xv[3])), rb);
                st_async16(dst + 16, make_uint4(__float_as_uint(xv[4]), __float_as_uint(xv[5]),
                                                __float_as_uint(xv[6]), __float_as_uint(xv[7])), rb);
            }
#pragma unroll
            for (int q = 0; q < kSwRhs; ++q) st_relaxed64(ll_own + r * kSwRhs + q, (1ull << 32) | __float_as_uint(xv[q]));
            if (r < bs) {
#pragma unroll
                for (int q = 0; q < kSwRhs; ++q)
                    if (q < ncg) a.Xr[(int64_t)(b0 + r) * a.ldr + cgc + q] = xv[q];
                if (a.upper) {  // the FP64 accumulation is off the chain
#pragma unroll
                    for (int q = 0; q < kSwRhs; ++q)
                        if (q < ncg) a.X64[(int64_t)(b0 + r) * a.ldx + cgc + q] += (double)xv[q];
                }
            }
        }
    } else {
        abandon();
    }
    cluster.sync();  // no CTA leaves while a push into its shared memory may be in flight
}

struct ReArgs {
    const double* A;
    int64_t lda;
    const double* X;
    int64_t ldx;
    const double* B;
    int64_t ldb;
    int n, nrhs;
    float* r32;          // P r in FP32 (row pinv[i] <- r_i)
    int64_t ldr;
    const int32_t* pinv;
    unsigned long long* nrm;  // [0,k) |r|, [k,2k) |x|, [2k,3k) |b|, [3k,4k) |d| (the correction just applied)
};

// r = b - A x for rows [64 blockIdx.x, +64) and columns [16 blockIdx.y, +16).  A and X stream
// through a 3-stage cp.async pipeline (64 x 64 tiles of A, 64 x 16 of X).  The products run on the
// FP64 tensor cores (mma.sync m16n8k4): warp w owns rows 16 (w % 4) .. +16 and the K half w / 4 of
// every chunk, and both 8-column tiles, so each A fragment feeds two MMAs.  Fragments
// (g = lane / 4, t = lane % 4): a = (A[g][k+t], A[g+8][k+t]), b = X[k+t][g],
// c = (C[g][2t], C[g][2t+1], C[g+8][2t], C[g+8][2t+1]).  Row strides of 66 (A) and 20 (X) doubles
// keep both fragment loads at two shared-memory wavefronts per warp.
__global__ void __launch_bounds__(256, 1) resid_kernel(ReArgs a) {
    extern __shared__ __align__(16) double re_sm[];
    __shared__ unsigned long long s_n[4 * kReRhs];
    const int t = threadIdx.x;
    const int r0 = blockIdx.x * kReRows, cb = blockIdx.y * kReRhs;
    const int nc = min(kReRhs, a.nrhs - cb);
    const int lane = t & 31, wp = t >> 5, mt = wp & 3, kh = wp >> 2, gq = lane >> 2, tq = lane & 3;
    const int nk = (int)ceil_div(a.n, kReK);
    if (t < 4 * kReRhs) s_n[t] = 0ull;
    auto issue = [&](int kc) {
        double* sa = re_sm + (kc % kReStages) * kReStage;
        double* sx = sa + kReRows * kReAS;
        const int k0 = kc * kReK;
#pragma unroll
        for (int i = 0; i < 8; ++i) {  // A: 64 rows x 32 pieces of 2 doubles
            const int piece = t + 256 * i, row = piece >> 5, kp = (piece & 31) * 2;
            const int grow = r0 + row, gk = k0 + kp;
            const bool ok = grow < a.n && gk < a.n;
            const double* src = ok ? a.A + (int64_t)grow * a.lda + gk : a.A;
            cp_async16(sa + row * kReAS + kp, src, ok ? (gk + 1 < a.n ? 16 : 8) : 0);
        }
#pragma unroll
        for (int i = 0; i < 2; ++i) {  // X: 64 k x 8 pieces of 2 doubles
            const int piece = t + 256 * i, k = piece >> 3, cp = (piece & 7) * 2;
            const int gk = k0 + k;
            const bool ok = gk < a.n && cp < nc;
            const double* src = ok ? a.X + (int64_t)gk * a.ldx + cb + cp : a.X;
            cp_async16(sx + k * kReXS + cp, src, ok ? (cp + 1 < nc ? 16 : 8) : 0);
        }
    };
    double d0[4] = {0.0, 0.0, 0.0, 0.0}, d1[4] = {0.0, 0.0, 0.0, 0.0};  // column tiles 0-7 and 8-15
#pragma unroll
    for (int s = 0; s < kReStages - 1; ++s) {
        if (s < nk) issue(s);
        cp_async_commit();
    }
    for (int kc = 0; kc < nk; ++kc) {
        cp_async_wait<kReStages - 2>();
        __syncthreads();
        if (kc + kReStages - 1 < nk) issue(kc + kReStages - 1);
        cp_async_commit();
        const double* sa = re_sm + (kc % kReStages) * kReStage;
        const double* sx = sa + kReRows * kReAS;
        const double* ra = sa + (16 * mt + gq) * kReAS + tq;
        const double* xb = sx + tq * kReXS + gq;
#pragma unroll
        for (int kk = 0; kk < kReK / kReSplit; kk += 4) {
            const int k = kh * (kReK / kReSplit) + kk;
            const double a0 = ra[k], a1 = ra[8 * kReAS + k];
            const double b0 = xb[k * kReXS], b1 = xb[k * kReXS + 8];
            asm volatile(
                "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
                : "+d"(d0[0]), "+d"(d0[1]), "+d"(d0[2]), "+d"(d0[3])
                : "d"(a0), "d"(a1), "d"(b0));
            asm volatile(
                "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
                : "+d"(d1[0]), "+d"(d1[1]), "+d"(d1[2]), "+d"(d1[3])
                : "d"(a0), "d"(a1), "d"(b1));
        }
    }
    cp_async_wait<0>();
    // reduce the K halves through shared memory
    __syncthreads();
    double* red = re_sm;  // [kReSplit][kReRows][kReRhs]
    {
        double* ra = red + (kh * kReRows + 16 * mt + gq) * kReRhs + 2 * tq;
        ra[0] = d0[0];
        ra[1] = d0[1];
        ra[8 * kReRhs] = d0[2];
        ra[8 * kReRhs + 1] = d0[3];
        ra[8] = d1[0];
        ra[9] = d1[1];
        ra[8 * kReRhs + 8] = d1[2];
        ra[8 * kReRhs + 9] = d1[3];
    }
    __syncthreads();
#pragma unroll
    for (int o = 0; o < 4; ++o) {
        const int e = t + 256 * o, rl = e >> 4, c = e & 15;
        const int row = r0 + rl;
        if (row >= a.n || c >= nc) continue;
        double sum = 0.0;
#pragma unroll
        for (int p = 0; p < kReSplit; ++p) sum += red[(p * kReRows + rl) * kReRhs + c];
        const int64_t gc = cb + c;
        const double bv = a.B[(int64_t)row * a.ldb + gc];
        const double xv = a.X[(int64_t)row * a.ldx + gc];
        const double rv = bv - sum;
        // the slot still holds the correction d of the sweeps that produced X (d[pinv[row]]: every
        // element of d is read once over the grid), which becomes the forward-error estimate
        float* slot = &a.r32[(int64_t)a.pinv[row] * a.ldr + gc];
        const float dv = *slot;
        *slot = (float)rv;
        atomicMax(&s_n[3 * kReRhs + c], (unsigned long long)__double_as_longlong(fabs((double)dv)));
        atomicMax(&s_n[c], (unsigned long long)__double_as_longlong(fabs(rv)));
        atomicMax(&s_n[kReRhs + c], (unsigned long long)__double_as_longlong(fabs(xv)));
        atomicMax(&s_n[2 * kReRhs + c], (unsigned long long)__double_as_longlong(fabs(bv)));
    }
    __syncthreads();
    if (t < 4 * kReRhs) {
        const int which = t / kReRhs, c = t - which * kReRhs;
        if (c < nc) atomicMax(&a.nrm[which * a.nrhs + cb + c], s_n[t]);
    }
}

// Whether the chained sweep can run here, and how many of its clusters fit at once: one launch
// of it with no blocks to solve (every CTA is padding and only meets its cluster's barriers) as a
// cooperative cluster launch, outside any capture.  A launch error leaves the chained sweep off.
template <int CL>
int chain_probe_one(Ctx* ctx, cudaStream_t st, int* why) {
    cudaError_t e = cudaFuncSetAttribute(trsv_chain_kernel<CL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         chain_smem<CL>());
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        *why = 1000 + (int)e;
        return 0;
    }
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.gridDim = dim3((unsigned)CL);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = chain_smem<CL>();
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int clusters = 0;
    e = cudaOccupancyMaxActiveClusters(&clusters, trsv_chain_kernel<CL>, &cfg);
    if (e != cudaSuccess || clusters < 1) {
        (void)cudaGetLastError();
        *why = e != cudaSuccess ? 2000 + (int)e : 4000;
        return 0;
    }
    SwArgs sa{};
    sa.n = 0;  // no blocks: every CTA is padding
    sa.status = ctx->d_status;
    e = cudaLaunchKernelEx(&cfg, trsv_chain_kernel<CL>, sa, CL);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        *why = 3000 + (int)e;
        return 0;
    }
    ctx->launches++;
    return clusters;
}

// Whether the chained sweep can run here, and how many of its clusters (of 8 and of 4 CTAs) fit at
// once: one launch of each with no blocks to solve (every CTA is padding and only meets its
// cluster's barriers) as a cooperative cluster launch, outside any capture.  A launch error leaves
// that cluster size off.
int32_t chain_probe(Ctx* ctx, cudaStream_t st) {
    if (ctx->chain_clusters >= 0) return B2M_OK;
    int why8 = 0, why4 = 0;
    ctx->chain_clusters = chain_probe_one<8>(ctx, st, &why8);
    ctx->chain_clusters4 = chain_probe_one<4>(ctx, st, &why4);
    ctx->chain_probe_why = (ctx->chain_clusters > 0 || ctx->chain_clusters4 > 0) ? 0 : (why8 ? why8 : why4);
    return B2M_OK;
}

// FP32 solve of the refinement: Xr (already permuted) <- U^-1 L^-1 Xr, X64 += Xr.
int32_t ir_solve(Ctx* ctx, cudaStream_t st, const float* LU, int64_t ld, int64_t n, const F32Scratch& s, float* Xr,
                 int64_t ldr, int64_t nrhs, double* X64, int64_t ldx) {
    const int nblk = (int)ceil_div(n, kTrsvNB);
    if (ctx->sweep_ctas < 0) {
        int per_sm = 0, coop = 0;
        B2M_CU(ctx, cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, ctx->device));
        B2M_CU(ctx, cudaFuncSetAttribute(trsv_sweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSwSmem));
        B2M_CU(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trsv_sweep_kernel, 256, kSwSmem));
        ctx->sweep_ctas = coop ? per_sm * ctx->num_sms : 0;
    }
    const int coop_ctas = ctx->sweep_ctas;
    for (int64_t c0 = 0; c0 < nrhs; c0 += kTrMaxRhs) {
        const int nc = (int)std::min<int64_t>(kTrMaxRhs, nrhs - c0);
        const int ng = (int)ceil_div(nc, kSwRhs);
        const int nbp8 = (int)round_up(nblk, 8), nbp4 = (int)round_up(nblk, 4);
        const int chain = ng > kSweepGroups ? 0
                          : ng * nbp8 / 8 <= ctx->chain_clusters ? 8
                          : ng * nbp4 / 4 <= ctx->chain_clusters4 ? 4 : 0;
        if (chain) {
            const int nbp = chain == 8 ? nbp8 : nbp4;
            // chained sweeps on clusters: one cooperative launch each
            for (int up = 0; up < 2; ++up) {
                const size_t ll_words = (size_t)nblk * ng * kTrsvNB * kSwRhs;
                unsigned long long* ll = s.ll + up * (size_t)nblk * kSweepGroups * kTrsvNB * kSwRhs;
                B2M_CU(ctx, cudaMemsetAsync(ll, 0, ll_words * sizeof(unsigned long long), st));
                SwArgs sa{LU,  ld, (int)n, up ? s.uinv : s.linv, up ? s.wu : s.wl, Xr, ldr, (int)c0, nc, X64, ldx, up,
                          ll, ctx->d_status, ctx->wait_limit >= 0 ? (uint32_t)ctx->wait_limit : kSwSpin};
                cudaLaunchConfig_t cfg{};
                cudaLaunchAttribute at[1];
                at[0].id = cudaLaunchAttributeCooperative;
                at[0].val.cooperative = 1;
                cfg.gridDim = dim3((unsigned)(nbp * ng));
                cfg.blockDim = dim3(256);
                cfg.dynamicSmemBytes = chain == 8 ? chain_smem<8>() : chain_smem<4>();
                cfg.stream = st;
                cfg.attrs = at;
                cfg.numAttrs = 1;
                prof_begin(ctx, st, kClsSolve);
                if (chain == 8) B2M_CU(ctx, cudaLaunchKernelEx(&cfg, trsv_chain_kernel<8>, sa, nbp));
                else B2M_CU(ctx, cudaLaunchKernelEx(&cfg, trsv_chain_kernel<4>, sa, nbp));
                prof_end(ctx, st, kClsSolve, 4.0 * (double)n * n / 2 + 4.0 * nblk * kTrsvNB * kTrsvNB + 8.0 * n * nc);
                B2M_LAUNCHED(ctx);
            }
            continue;
        }
        if (nblk * ng <= coop_ctas && ng <= kSweepGroups) {
            // persistent sweeps: one cooperative launch each
            for (int up = 0; up < 2; ++up) {
                const size_t ll_words = (size_t)nblk * ng * kTrsvNB * kSwRhs;
                unsigned long long* ll = s.ll + up * (size_t)nblk * kSweepGroups * kTrsvNB * kSwRhs;
                B2M_CU(ctx, cudaMemsetAsync(ll, 0, ll_words * sizeof(unsigned long long), st));
                SwArgs sa{LU,  ld, (int)n, up ? s.uinv : s.linv, up ? s.wu : s.wl, Xr, ldr, (int)c0, nc, X64, ldx, up,
                          ll, ctx->d_status, ctx->wait_limit >= 0 ? (uint32_t)ctx->wait_limit : kSwSpin};
                cudaLaunchConfig_t cfg{};
                cudaLaunchAttribute at[1];
                at[0].id = cudaLaunchAttributeCooperative;
                at[0].val.cooperative = 1;
                cfg.gridDim = dim3((unsigned)(nblk * ng));
                cfg.blockDim = dim3(256);
                cfg.dynamicSmemBytes = kSwSmem;
                cfg.stream = st;
                cfg.attrs = at;
                cfg.numAttrs = 1;
                prof_begin(ctx, st, kClsSolve);
                B2M_CU(ctx, cudaLaunchKernelEx(&cfg, trsv_sweep_kernel, sa));
                prof_end(ctx, st, kClsSolve, 4.0 * (double)n * n / 2 + 4.0 * nblk * kTrsvNB * kTrsvNB + 8.0 * n * nc);
                B2M_LAUNCHED(ctx);
            }
            continue;
        }
        TrArgs a{LU, ld, (int)n, s.linv, Xr, ldr, (int)c0, nc, X64, ldx, 0, (int)ceil_div(nc, kTrRhs), ctx->d_status};
        for (int b = 0; b < nblk; ++b) {
            const int rows = (int)(n - std::min<int64_t>(n, (int64_t)(b + 1) * kTrsvNB));
            const int nu = b > 0 ? (int)ceil_div(rows, kTrRows) : 0;
            prof_begin(ctx, st, kClsSolve);
            trsv_block_kernel<<<a.nd + nu, 256, 0, st>>>(a, b);
            prof_end(ctx, st, kClsSolve, 4.0 * kTrsvNB * (rows + kTrsvNB) + 8.0 * (rows + kTrsvNB) * nc);
            B2M_LAUNCHED(ctx);
        }
        a.upper = 1;
        a.inv = s.uinv;
        for (int b = nblk - 1; b >= 0; --b) {
            const int rows = b * kTrsvNB;
            const int nu = b < nblk - 1 ? (int)ceil_div(rows, kTrRows) : 0;
            prof_begin(ctx, st, kClsSolve);
            trsv_block_kernel<<<a.nd + nu, 256, 0, st>>>(a, b);
            prof_end(ctx, st, kClsSolve, 4.0 * kTrsvNB * (rows + kTrsvNB) + 8.0 * (rows + kTrsvNB) * nc);
            B2M_LAUNCHED(ctx);
        }
    }
    return B2M_OK;
}

double eta_from(const std::vector<unsigned long long>& h, int64_t nrhs, double normA) {
    double eta = 0.0;
    for (int64_t c = 0; c < nrhs; ++c) {
        const double rn = __builtin_bit_cast(double, h[c]);
        const double xn = __builtin_bit_cast(double, h[nrhs + c]);
        const double bn = __builtin_bit_cast(double, h[2 * nrhs + c]);
        const double den = normA * xn + bn;
        eta = std::max(eta, den > 0 ? rn / den : (rn > 0 ? INFINITY : 0.0));
    }
    return eta;
}

// forward-error estimate max_c ||e_c||inf / ||x_c||inf from the column maxima [k,2k) |x| and
// [3k,4k) |d| of the last correction d.  d_k is (to first order) the error of the iterate before
// it, so ||d_k|| alone overstates the error of x_k by the contraction factor; with the previous
// step's ||d_(k-1)|| (dprev, < 0 when there is none) the error of x_k is estimated as
// ||d_k|| * rho with rho = ||d_k|| / ||d_(k-1)|| (linear convergence), and as ||d_k|| otherwise.
// dprev is updated to this step's ||d_c||.
double fwd_from(const std::vector<unsigned long long>& h, int64_t nrhs, std::vector<double>* dprev = nullptr) {
    double f = 0.0;
    for (int64_t c = 0; c < nrhs; ++c) {
        const double xn = __builtin_bit_cast(double, h[nrhs + c]);
        const double dn = __builtin_bit_cast(double, h[3 * nrhs + c]);
        double rho = 1.0;
        if (dprev && (*dprev)[c] > 0.0) rho = std::min(1.0, dn / (*dprev)[c]);
        if (dprev) (*dprev)[c] = dn;
        f = std::max(f, xn > 0 ? dn * rho / xn : (dn > 0 ? INFINITY : 0.0));
    }
    return f;
}

}  // namespace

// ------------------------------------------------------------------ the refinement driver
int32_t solve_mixed(Ctx* ctx, cudaStream_t st, const double* A, int64_t lda, int64_t n, const double* B, int64_t ldb,
                    double* X, int64_t ldx, int64_t nrhs, int mode, int max_iter, double tol, MixedReport* rep) {
    if (mode != 1 && mode != 3) return fail(ctx, B2M_ERR_ARG, "mode must be 1 (TF32) or 3 (3xTF32)");
    if ((lda & 1) || (ldb & 1) || (ldx & 1) || !aligned16(A) || !aligned16(B) || !aligned16(X))
        return fail(ctx, B2M_ERR_DIM, "solve_mixed: device operands need even strides and 16-byte alignment");
    const int64_t ld32 = round_up(n, 32);
    const int64_t ldr = round_up(nrhs, 4);
    // workspace layout: [A32 | factorisation scratch] kWsMatD, [r32] kWsE, [perm | pinv] kWsPiv,
    // norms kWsSmall
    const size_t a32_bytes = (size_t)round_up(n * ld32 * (int64_t)sizeof(float), 256);
    void *pD, *pE, *pP, *pS;
    B2M_TRY(ws_get(ctx, kWsMatD, a32_bytes + f32_scratch_bytes(n), &pD));
    B2M_TRY(ws_get(ctx, kWsE, (size_t)(n * ldr) * sizeof(float), &pE));
    B2M_TRY(ws_get(ctx, kWsPiv, (size_t)(2 * n) * sizeof(int32_t), &pP));
    B2M_TRY(ws_get(ctx, kWsSmall, (size_t)(4 + 4 * nrhs) * sizeof(unsigned long long), &pS));
    float* A32 = (float*)pD;
    const F32Scratch sc = f32_scratch_carve(static_cast<char*>(pD) + a32_bytes, n);
    float* r32 = (float*)pE;
    int32_t* perm = (int32_t*)pP;
    int32_t* pinv = perm + n;
    unsigned long long* nrm = (unsigned long long*)pS;
    std::vector<unsigned long long> h((size_t)(1 + 4 * nrhs));

    MixedReport local{};
    if (!rep) rep = &local;
    *rep = MixedReport{};
    std::atomic<int>& attr = device_flag((const void*)resid_kernel, 0, ctx->device);
    if (!attr.load()) {
        B2M_CU(ctx, cudaFuncSetAttribute(resid_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kReSmem));
        attr.store(1);
    }

    B2M_CU(ctx, cudaMemsetAsync(ctx->d_status, 0, kNumStatus * sizeof(int32_t), st));
    B2M_CU(ctx, cudaMemsetAsync(nrm, 0, sizeof(unsigned long long), st));
    f64_to_f32_norm_kernel<<<(unsigned)std::min<int64_t>(ceil_div(n, 8), 8 * ctx->num_sms), 256, 0, st>>>(
        A, lda, A32, ld32, n, nrm);
    B2M_LAUNCHED(ctx);
    B2M_TRY(chain_probe(ctx, st));
    B2M_TRY(lu_factor_f32(ctx, st, A32, ld32, n, perm, mode, sc));
    B2M_CU(ctx, cudaMemcpyAsync(ctx->h_status, ctx->d_status, kNumStatus * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    B2M_CU(ctx, cudaMemcpyAsync(h.data(), nrm, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    B2M_CU(ctx, cudaStreamSynchronize(st));
    if (ctx->h_status[kTimeout]) return fail(ctx, B2M_ERR_TIMEOUT, "bounded wait gave up (site %d)", ctx->h_status[kTimeout]);
    const double normA = __builtin_bit_cast(double, h[0]);

    bool converged = false;
    if (ctx->h_status[kInfo] == 0) {
        invert_perm_kernel<<<gsz(n), 256, 0, st>>>(perm, pinv, n);
        B2M_LAUNCHED(ctx);
        ir_init_kernel<<<gsz(n * nrhs), 256, 0, st>>>(B, ldb, perm, r32, ldr, X, ldx, n, nrhs);
        B2M_LAUNCHED(ctx);
        // one refinement step: d = (LU)^-1 P r in FP32, x += d, r = b - A x in FP64 (and P r in FP32)
        const GraphKey key{5 + mode * 10, A32, X, B, A, ld32, n, nrhs, lda * 1000003 + ldb * 1009 + ldx};
        auto step = [&](cudaStream_t q) -> int32_t {
            B2M_TRY(ir_solve(ctx, q, A32, ld32, n, sc, r32, ldr, nrhs, X, ldx));
            B2M_CU(ctx, cudaMemsetAsync(nrm + 1, 0, 4 * nrhs * sizeof(unsigned long long), q));
            ReArgs ra{A, lda, X, ldx, B, ldb, (int)n, (int)nrhs, r32, ldr, pinv, nrm + 1};
            prof_begin(ctx, q, kClsOther);
            resid_kernel<<<dim3((unsigned)ceil_div(n, kReRows), (unsigned)ceil_div(nrhs, kReRhs)), 256, kReSmem, q>>>(ra);
            prof_end(ctx, q, kClsOther, 8.0 * n * n + 8.0 * 3 * n * nrhs);  // bytes: A once, B, X, r
            B2M_LAUNCHED(ctx);
            return B2M_OK;
        };
        double prev = INFINITY;
        std::vector<double> dprev((size_t)nrhs, -1.0);
        for (int it = 0; it < max_iter; ++it) {
            B2M_TRY(run_graph(ctx, st, key, step));
            B2M_CU(ctx, cudaMemcpyAsync(h.data() + 1, nrm + 1, 4 * nrhs * sizeof(unsigned long long),
                                        cudaMemcpyDeviceToHost, st));
            B2M_CU(ctx, cudaMemcpyAsync(ctx->h_status, ctx->d_status, kNumStatus * sizeof(int32_t),
                                        cudaMemcpyDeviceToHost, st));
            B2M_CU(ctx, cudaStreamSynchronize(st));
            // a sweep wait that gave up leaves X unfinished: that is an error, not a stall, and the
            // fallback below (which clears the status words) must not hide it
            if (ctx->h_status[kTimeout])
                return fail(ctx, B2M_ERR_TIMEOUT, "bounded wait gave up in refinement step %d (site %d)", it + 1,
                            ctx->h_status[kTimeout]);
            std::vector<unsigned long long> hv(h.begin() + 1, h.end());
            const double eta = eta_from(hv, nrhs, normA);
            rep->iterations = it + 1;
            rep->backward_error = eta;
            rep->ir_backward_error = eta;
            rep->forward_error = fwd_from(hv, nrhs, &dprev);
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
    B2M_TRY(ws_get(ctx, kWsSmall, (size_t)(4 + 4 * nrhs) * sizeof(unsigned long long), &pS));
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
        B2M_CU(ctx, cudaMemsetAsync(nrm, 0, (1 + 4 * nrhs) * sizeof(unsigned long long), st));
        norm_inf_kernel<<<gsz(n, 8), 256, 0, st>>>(A, lda, n, nrm);
        B2M_LAUNCHED(ctx);
        colmax3_kernel<<<gsz(n * nrhs), 256, 0, st>>>(R, ldr, X, ldx, B, ldb, n, nrhs, nrm + 1);
        B2M_LAUNCHED(ctx);
        // forward-error estimate: one more correction d = (LU)^-1 r with the FP64 factors
        B2M_TRY(lu_solve_f64(ctx, st, LU, ld, n, ipiv + n, R, ldr, nrhs));
        colmax_kernel<<<gsz(n * nrhs), 256, 0, st>>>(R, ldr, n, nrhs, nrm + 1 + 3 * nrhs);
        B2M_LAUNCHED(ctx);
        std::vector<unsigned long long> h((size_t)(1 + 4 * nrhs));
        B2M_CU(ctx, cudaMemcpyAsync(h.data(), nrm, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        B2M_CU(ctx, cudaStreamSynchronize(st));
        const double normA = __builtin_bit_cast(double, h[0]);
        std::vector<unsigned long long> hv(h.begin() + 1, h.end());
        rep->backward_error = eta_from(hv, nrhs, normA);
        rep->forward_error = fwd_from(hv, nrhs);
    }
    return B2M_OK;
}

}  // namespace b2m
