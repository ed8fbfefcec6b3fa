// dgemm.cu -- FP64 GEMM on the sm_100a DMMA path (mma.sync m16n8k4 .f64), operands staged by
// TMA into a multi-stage shared-memory ring guarded by mbarriers (one producer warp, eight
// consumer warps).  Replaces the reference's BlockMatrixMultiplication(T1/T2) + the FMA
// MatrixMultT2 inner kernel (BlockedMult.pas:350-724, FMAMatrixMultTransposedOperationsx64.pas)
// and applies the doNone/doAdd/doSub destination operation (MatrixConst.pas:147) in the epilogue.
//
// CTA tile 128 x 128, k-step 16 doubles, 6 stages (192 KiB).  A K-major tile ([m][k], k
// contiguous) is loaded with the 128-byte swizzle, which makes the per-thread fragment loads
// conflict-free; an MN-major tile ([k][m or n]) is loaded unswizzled (one 1 KiB row per k).
#include "common.cuh"
#include "kernels.cuh"

namespace b2m {
namespace {

constexpr int BM = 128, BN = 128, BKD = 16, STAGES = 6;
constexpr int kConsumerWarps = 8;
constexpr int kThreads = (kConsumerWarps + 1) * 32;
constexpr int kTileBytes = BM * BKD * 8;          // 16 KiB per operand tile
constexpr int kStageBytes = 2 * kTileBytes;
constexpr int kSmemBytes = STAGES * kStageBytes + 1024;
constexpr int kGroupM = 8;

struct DgemmArgs {
    int M, N, K;
    int a_x0, a_y0, b_x0, b_y0;
    double* C;
    int64_t ldc;
    int op;
    int32_t* status;
    int check_info;
};

__device__ __forceinline__ void dmma16x8x4(double (&d)[4], double a0, double a1, double b0) {
    asm volatile(
        "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};\n"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a0), "d"(a1), "d"(b0));
}

__device__ __forceinline__ double lds64(const uint8_t* base, uint32_t off) {
    return *reinterpret_cast<const double*>(base + off);
}

template <bool AK, bool BKM>
__global__ void __launch_bounds__(kThreads, 1)
    dgemm_tma_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, DgemmArgs p) {
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[STAGES];
    __shared__ __align__(8) uint64_t empty_bar[STAGES];

    if (p.check_info && p.status[kInfo] != 0) return;  // an earlier singular pivot stops the chain

    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));

    const int tiles_m = (p.M + BM - 1) / BM;
    const int tiles_n = (p.N + BN - 1) / BN;
    const int bid = blockIdx.x;
    const int group = bid / (kGroupM * tiles_n);
    const int first_m = group * kGroupM;
    const int gsize = min(tiles_m - first_m, kGroupM);
    const int in_group = bid % (kGroupM * tiles_n);
    const int tm = first_m + in_group % gsize;
    const int tn = in_group / gsize;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int KT = (p.K + BKD - 1) / BKD;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], kConsumerWarps);
        }
        fence_barrier_init();
    }
    __syncthreads();

    if (warp == kConsumerWarps) {
        // ---------------- producer: one elected lane issues the TMA loads
        if (lane == 0) {
            tma_prefetch_desc(&tmA);
            tma_prefetch_desc(&tmB);
            for (int kt = 0; kt < KT; ++kt) {
                const int s = kt % STAGES;
                const uint32_t ph = (kt / STAGES) & 1;
                if (!mbar_wait(&empty_bar[s], ph ^ 1, &p.status[kTimeout], 101)) break;
                uint8_t* sa = smem + s * kStageBytes;
                uint8_t* sb = sa + kTileBytes;
                mbar_arrive_expect_tx(&full_bar[s], kStageBytes);
                if (AK) tma_load_2d(sa, &tmA, p.a_x0 + kt * BKD, p.a_y0 + tm * BM, &full_bar[s]);
                else    tma_load_2d(sa, &tmA, p.a_x0 + tm * BM, p.a_y0 + kt * BKD, &full_bar[s]);
                if (BKM) tma_load_2d(sb, &tmB, p.b_x0 + kt * BKD, p.b_y0 + tn * BN, &full_bar[s]);
                else     tma_load_2d(sb, &tmB, p.b_x0 + tn * BN, p.b_y0 + kt * BKD, &full_bar[s]);
            }
        }
        return;
    }

    // ---------------- consumers: 2 (m) x 4 (n) warps, warp tile 64 x 32
    const int wm = warp >> 2, wn = warp & 3;
    const int g = lane >> 2, t = lane & 3;

    // per-thread fragment offsets (bytes within a stage tile), k4-step 0
    uint32_t offA[4], offB[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int m = wm * 64 + i * 16 + g;
        offA[i] = AK ? (uint32_t)(m * 128 + ((t & 1) << 3)) : (uint32_t)(t * 1024 + m * 8);
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int n = wn * 32 + j * 8 + g;
        offB[j] = BKM ? (uint32_t)(n * 128 + ((t & 1) << 3)) : (uint32_t)(t * 1024 + n * 8);
    }

    double acc[4][4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0;

    bool ok = true;
    for (int kt = 0; kt < KT; ++kt) {
        const int s = kt % STAGES;
        const uint32_t ph = (kt / STAGES) & 1;
        if (!mbar_wait(&full_bar[s], ph, &p.status[kTimeout], 102)) { ok = false; break; }
        const uint8_t* sa = smem + s * kStageBytes;
        const uint8_t* sb = sa + kTileBytes;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            double a0[4], a1[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                if (AK) {
                    const uint32_t o = offA[i] + ((((2 * q + (t >> 1)) ^ g) & 7) << 4);
                    a0[i] = lds64(sa, o);
                    a1[i] = lds64(sa, o + 1024);
                } else {
                    const uint32_t o = offA[i] + q * 4 * 1024;
                    a0[i] = lds64(sa, o);
                    a1[i] = lds64(sa, o + 64);
                }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (BKM) b[j] = lds64(sb, offB[j] + ((((2 * q + (t >> 1)) ^ g) & 7) << 4));
                else     b[j] = lds64(sb, offB[j] + q * 4 * 1024);
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma16x8x4(acc[i][j], a0[i], a1[i], b[j]);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty_bar[s]);
    }
    if (!ok) return;

    // ---------------- epilogue: dest op= acc, masked to the M x N operand
    const int m_base = tm * BM + wm * 64;
    const int n_base = tn * BN + wn * 32;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int m = m_base + i * 16 + g + h * 8;
            if (m >= p.M) continue;
            double* crow = p.C + (int64_t)m * p.ldc;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int n = n_base + j * 8 + 2 * t + e;
                    if (n >= p.N) continue;
                    const double v = acc[i][j][2 * h + e];
                    if (p.op == B2M_DO_NONE) crow[n] = v;
                    else if (p.op == B2M_DO_ADD) crow[n] = crow[n] + v;
                    else crow[n] = crow[n] - v;
                }
            }
        }
    }
}

template <bool AK, bool BKM>
int32_t launch_variant(Ctx* ctx, cudaStream_t st, const CUtensorMap& ta, const CUtensorMap& tb, const DgemmArgs& a) {
    std::atomic<int>& attr_set = device_flag((const void*)dgemm_tma_kernel<AK, BKM>, 0, ctx->device);
    if (!attr_set.load()) {
        B2M_CU(ctx, cudaFuncSetAttribute(dgemm_tma_kernel<AK, BKM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kSmemBytes));
        attr_set.store(1);
    }
    const int tiles = (int)(ceil_div(a.M, BM) * ceil_div(a.N, BN));
    prof_begin(ctx, st, kClsGemm);
    B2M_CU(ctx, launch_k(ctx, dgemm_tma_kernel<AK, BKM>, dim3(tiles), dim3(kThreads), kSmemBytes, st, ta, tb, a));
    prof_end(ctx, st, kClsGemm, 2.0 * a.M * a.N * a.K);
    B2M_LAUNCHED(ctx);
    return B2M_OK;
}

// C op= A(:, k0:k0+kt) B(k0:k0+kt, :) for a short k range (kt < 16): the tail of a K that ends inside
// the operands' tensor maps, where the 16-wide TMA k-tile would read other data.  One thread per
// output, K FMAs each; these tails are narrow (the 8-column leaves of very tall factorisations).
__global__ void dgemm_ktail_kernel(const double* A, int64_t lda, int64_t ar0, int64_t ac0, int akmajor,
                                   const double* B, int64_t ldb, int64_t br0, int64_t bc0, int bkmajor, double* C,
                                   int64_t ldc, int M, int N, int k0, int kt, int op, const int32_t* status,
                                   int check_info) {
    if (check_info && status[kInfo] != 0) return;
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)M * N) return;
    const int m = (int)(e / N), n = (int)(e - (int64_t)m * N);
    double s = 0.0;
    for (int k = k0; k < k0 + kt; ++k) {
        const double a = akmajor ? A[(ar0 + m) * lda + ac0 + k] : A[(ar0 + k) * lda + ac0 + m];
        const double b = bkmajor ? B[(br0 + n) * ldb + bc0 + k] : B[(br0 + k) * ldb + bc0 + n];
        s = fma(a, b, s);
    }
    double* c = C + (int64_t)m * ldc + n;
    *c = op == B2M_DO_NONE ? s : (op == B2M_DO_ADD ? *c + s : *c - s);
}

}  // namespace

int32_t dgemm_tiled(Ctx* ctx, cudaStream_t st, const DOperand& A, const DOperand& B, double* C, int64_t ldc, int64_t M,
                    int64_t N, int64_t K, int op, bool check_info) {
    if (M <= 0 || N <= 0) return B2M_OK;
    if (K <= 0) {
        if (op == B2M_DO_NONE) B2M_CU(ctx, cudaMemset2DAsync(C, ldc * 8, 0, N * 8, M, st));
        return B2M_OK;
    }
    // A K that is not a multiple of the 16-wide k-tile is safe only where the k range ends at the
    // tensor maps' extent (TMA fills beyond it with zeros); elsewhere the last partial k-tile runs
    // as a separate short-K pass after the tiled product of the first K - K % 16.
    const int64_t a_kend = A.kmajor ? A.c0 + K : A.r0 + K, a_ext = A.kmajor ? A.cols : A.rows;
    const int64_t b_kend = B.kmajor ? B.c0 + K : B.r0 + K, b_ext = B.kmajor ? B.cols : B.rows;
    if ((K & 15) && (a_kend != a_ext || b_kend != b_ext)) {
        const int64_t K16 = K & ~int64_t(15);
        int tail_op = op;
        if (K16 > 0) {
            B2M_TRY(dgemm_tiled(ctx, st, A, B, C, ldc, M, N, K16, op, check_info));
            if (op == B2M_DO_NONE) tail_op = B2M_DO_ADD;
        }
        const int64_t outs = M * N;
        prof_begin(ctx, st, kClsGemm);
        B2M_CU(ctx, launch_k(ctx, dgemm_ktail_kernel, dim3((unsigned)ceil_div(outs, 256)), dim3(256), 0, st,
                             static_cast<const double*>(A.base), A.ld, A.r0, A.c0, A.kmajor ? 1 : 0,
                             static_cast<const double*>(B.base), B.ld, B.r0, B.c0, B.kmajor ? 1 : 0, C, ldc, (int)M,
                             (int)N, (int)K16, (int)(K - K16), tail_op, ctx->d_status, check_info ? 1 : 0));
        prof_end(ctx, st, kClsGemm, 2.0 * M * N * (K - K16));
        B2M_LAUNCHED(ctx);
        return B2M_OK;
    }
    if ((A.c0 & 1) || (B.c0 & 1) || (A.ld & 1) || (B.ld & 1))
        return fail(ctx, B2M_ERR_DIM, "dgemm_tiled: TMA origin/stride must be even (A.c0=%lld B.c0=%lld)",
                    (long long)A.c0, (long long)B.c0);
    CUtensorMap ta, tb;
    if (A.kmajor)
        B2M_TRY(encode_tmap_2d(ctx, &ta, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, A.base, A.cols, A.rows, A.ld * 8, BKD, BM,
                               CU_TENSOR_MAP_SWIZZLE_128B));
    else
        B2M_TRY(encode_tmap_2d(ctx, &ta, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, A.base, A.cols, A.rows, A.ld * 8, BM, BKD,
                               CU_TENSOR_MAP_SWIZZLE_NONE));
    if (B.kmajor)
        B2M_TRY(encode_tmap_2d(ctx, &tb, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, B.base, B.cols, B.rows, B.ld * 8, BKD, BN,
                               CU_TENSOR_MAP_SWIZZLE_128B));
    else
        B2M_TRY(encode_tmap_2d(ctx, &tb, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, B.base, B.cols, B.rows, B.ld * 8, BN, BKD,
                               CU_TENSOR_MAP_SWIZZLE_NONE));
    DgemmArgs a;
    a.M = (int)M; a.N = (int)N; a.K = (int)K;
    a.a_x0 = (int)A.c0; a.a_y0 = (int)A.r0;
    a.b_x0 = (int)B.c0; a.b_y0 = (int)B.r0;
    a.C = C; a.ldc = ldc; a.op = op;
    a.status = ctx->d_status;
    a.check_info = check_info ? 1 : 0;
    if (A.kmajor && !B.kmajor) return launch_variant<true, false>(ctx, st, ta, tb, a);
    if (A.kmajor && B.kmajor) return launch_variant<true, true>(ctx, st, ta, tb, a);
    if (!A.kmajor && !B.kmajor) return launch_variant<false, false>(ctx, st, ta, tb, a);
    return launch_variant<false, true>(ctx, st, ta, tb, a);
}

}  // namespace b2m
