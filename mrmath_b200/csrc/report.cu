// report.cu -- error reports of GEMM results against compensated products.
//
// No counterpart in the reference, whose MatrixMult returns nothing but the product.  A caller of
// the DMMA or Ozaki GEMM may ask how far its result is from the exact product: the report samples
// rows of the result and compares every entry of those rows with the product of the same operands
// summed with the Ogita-Rump-Oishi compensated dot product (Dot2: TwoProduct by FMA, TwoSum), which
// is as accurate as if computed in twice the working precision.  Reported, over the sampled rows:
//   forward_error   max_ij |C_ij - C*_ij| / max_ij (|A||B|)_ij   (the normwise quantity a GEMM's
//                   a-priori bound K u |A||B| speaks of)
//   relative_error  ||C - C*||_F / ||C*||_F
#include "common.cuh"
#include "kernels.cuh"

namespace b2m {
namespace {

constexpr int kRpThreads = 256;
constexpr int kRpKChunk = 1024;  // A row elements staged in shared memory per pass

struct RpArgs {
    const double* C;
    int64_t ldc;
    const double* A;  // element (m, k) = A[m * lda + k] (a_kmajor) or A[k * lda + m]
    int64_t lda;
    int a_kmajor;
    const double* B;  // element (k, n) = B[k * ldb + n] (b_nmajor) or B[n * ldb + k]
    int64_t ldb;
    int b_nmajor;
    int M, N, K, rows;
    double* acc;  // [0] max |C - C*| bits, [1] max |A||B| bits, [2] sum (C - C*)^2, [3] sum C*^2
};

__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
    s = a + b;
    const double z = s - a;
    e = (a - (s - z)) + (b - z);
}

// one CTA per (sampled row, 256-column block); the sampled row's A values pass through shared
// memory; CTAs of the same column block run together, so B's block is re-read from L2
__global__ void __launch_bounds__(kRpThreads) gemm_report_kernel(RpArgs p) {
    __shared__ double s_a[kRpKChunk];
    __shared__ double s_red[4][kRpThreads / 32];
    const int sr = blockIdx.x % p.rows;
    const int m = (int)(((int64_t)sr * p.M) / p.rows);
    const int n = (blockIdx.x / p.rows) * kRpThreads + threadIdx.x;
    double s = 0.0, comp = 0.0, abs_s = 0.0;
    for (int k0 = 0; k0 < p.K; k0 += kRpKChunk) {
        const int kc = min(kRpKChunk, p.K - k0);
        __syncthreads();
        for (int k = threadIdx.x; k < kc; k += kRpThreads)
            s_a[k] = p.a_kmajor ? p.A[(int64_t)m * p.lda + k0 + k] : p.A[(int64_t)(k0 + k) * p.lda + m];
        __syncthreads();
        if (n < p.N) {
            for (int k = 0; k < kc; ++k) {
                const double a = s_a[k];
                const double b = p.b_nmajor ? p.B[(int64_t)(k0 + k) * p.ldb + n] : p.B[(int64_t)n * p.ldb + k0 + k];
                const double prod = a * b;
                const double ep = fma(a, b, -prod);  // TwoProduct
                double t, et;
                two_sum(s, prod, t, et);
                s = t;
                comp += et + ep;
                abs_s = fma(fabs(a), fabs(b), abs_s);
            }
        }
    }
    double err = 0.0, ab = 0.0, e2 = 0.0, c2 = 0.0;
    if (n < p.N) {
        const double exact = s + comp;
        const double d = p.C[(int64_t)m * p.ldc + n] - exact;
        err = fabs(d);
        ab = abs_s;
        e2 = d * d;
        c2 = exact * exact;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        err = fmax(err, __shfl_xor_sync(0xffffffffu, err, o));
        ab = fmax(ab, __shfl_xor_sync(0xffffffffu, ab, o));
        e2 += __shfl_xor_sync(0xffffffffu, e2, o);
        c2 += __shfl_xor_sync(0xffffffffu, c2, o);
    }
    if (lane == 0) {
        s_red[0][warp] = err;
        s_red[1][warp] = ab;
        s_red[2][warp] = e2;
        s_red[3][warp] = c2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kRpThreads / 32; ++w) {
            err = fmax(err, s_red[0][w]);
            ab = fmax(ab, s_red[1][w]);
            e2 += s_red[2][w];
            c2 += s_red[3][w];
        }
        // non-negative doubles order like their bit patterns
        atomicMax(reinterpret_cast<unsigned long long*>(&p.acc[0]), (unsigned long long)__double_as_longlong(err));
        atomicMax(reinterpret_cast<unsigned long long*>(&p.acc[1]), (unsigned long long)__double_as_longlong(ab));
        atomicAdd(&p.acc[2], e2);
        atomicAdd(&p.acc[3], c2);
    }
}

}  // namespace

int32_t gemm_error_report(Ctx* ctx, cudaStream_t st, const double* C, int64_t ldc, const double* A, int64_t lda,
                          bool a_kmajor, const double* B, int64_t ldb, bool b_nmajor, int64_t M, int64_t N, int64_t K,
                          int rows, double* host_out4) {
    if (M <= 0 || N <= 0 || K <= 0 || rows <= 0) {
        for (int i = 0; i < 4; ++i) host_out4[i] = 0.0;
        return B2M_OK;
    }
    if (M > (1 << 30) || N > (1 << 30) || K > (1 << 30)) return fail(ctx, B2M_ERR_UNSUPPORTED, "report: too large");
    rows = (int)std::min<int64_t>(rows, M);
    void* p;
    B2M_TRY(ws_get(ctx, kWsH, 4 * sizeof(double), &p));
    double* acc = static_cast<double*>(p);
    B2M_CU(ctx, cudaMemsetAsync(acc, 0, 4 * sizeof(double), st));
    RpArgs a{C, ldc, A, lda, a_kmajor ? 1 : 0, B, ldb, b_nmajor ? 1 : 0, (int)M, (int)N, (int)K, rows, acc};
    const int64_t ctas = (int64_t)rows * ceil_div(N, kRpThreads);
    if (ctas > 0x7fffffff) return fail(ctx, B2M_ERR_UNSUPPORTED, "report: too many sampled entries");
    gemm_report_kernel<<<(unsigned)ctas, kRpThreads, 0, st>>>(a);
    B2M_LAUNCHED(ctx);
    B2M_CU(ctx, cudaMemcpyAsync(host_out4, acc, 4 * sizeof(double), cudaMemcpyDeviceToHost, st));
    B2M_CU(ctx, cudaStreamSynchronize(st));
    return B2M_OK;
}

}  // namespace b2m
