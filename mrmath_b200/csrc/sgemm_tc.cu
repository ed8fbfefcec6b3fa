// sgemm_tc.cu -- FP32 GEMM on the 5th-generation tensor cores (tcgen05.mma kind::tf32, accumulator in
// TMEM), the trailing-update GEMM of the mixed-precision LU.
//
//   C(M x N) op= A(M x K) * B(K x N),  A given K-major (row-major M x K), B given as Bt (N x K,
//   k contiguous), C row-major FP32; op = none / add / sub as the reference's destination ops.
//
// Precision modes: 1 = TF32 (the hardware reads the top 19 bits of each FP32 operand);
// 3 = 3xTF32: operands are pre-split as x = hi + lo with hi = x with its 13 low mantissa bits
// cleared, lo = x - hi (exact), and C accumulates hi*hi + hi*lo + lo*hi, which restores close to
// FP32 accuracy (relative error ~2^-21 per product instead of 2^-11).
//
// CTA: 6 warps.  Warps 0-3: epilogue (warp w reads TMEM lanes 32w..32w+31), warp 4: TMA producer,
// warp 5: TMEM allocation and the single MMA-issuing thread.  Tile 128 x 128, k-step 32 floats
// (one 128-byte swizzle row), 4 MMAs of K = 8 per k-step; stages guarded by mbarriers, smem
// stages released by tcgen05.commit.  Epilogue: TMEM -> registers -> 128-byte-swizzled staging
// tiles in the (then idle) stage memory -> TMA tensor store (op none) or TMA reduce-add (op add,
// and op sub with the accumulator negated), so C is never read by the SM and every global write
// is a full 128-byte line.
#include "common.cuh"
#include "kernels.cuh"

namespace b2m {
namespace {

constexpr int TBM = 128, TBN = 128, TBK = 32;
constexpr int kTileB = TBM * TBK * 4;  // 16 KiB per operand tile
constexpr int kTcThreads = 192;

struct TcArgs {
    int M, N, K;
    int c_x0, c_y0;
    int a_x0, a_y0, b_x0, b_y0;
    float* C;
    int64_t ldc;
    int op;
    int split;  // 1 or 3
    int32_t* status;
    int check_info;
};

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(dst)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void umma_tf32(uint32_t tmem_c, uint64_t da, uint64_t db, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_c),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     smem_u32(bar))
                 : "memory");
}
// K-major operand tile in shared memory, 128-byte swizzle: rows of 128 B, 8-row groups 1024 B apart
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}
// tf32 x tf32 -> f32, both K-major, M = 128, N = TBN
__host__ __device__ constexpr uint32_t tf32_idesc() {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TBN >> 3) << 17) | ((uint32_t)(TBM >> 4) << 24);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

template <int SPLIT>
__global__ void __launch_bounds__(kTcThreads, 1)
    sgemm_tc_kernel(const __grid_constant__ CUtensorMap tmAh, const __grid_constant__ CUtensorMap tmAl,
                    const __grid_constant__ CUtensorMap tmBh, const __grid_constant__ CUtensorMap tmBl,
                    const __grid_constant__ CUtensorMap tmC, TcArgs p) {
    constexpr int NOPS = SPLIT == 3 ? 4 : 2;            // operand tiles per stage
    constexpr int STAGES = SPLIT == 3 ? 3 : 5;
    constexpr int kStage = NOPS * kTileB;
    extern __shared__ uint8_t tc_smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[STAGES];
    __shared__ __align__(8) uint64_t empty_bar[STAGES];
    __shared__ __align__(8) uint64_t acc_bar;
    __shared__ uint32_t tmem_base_sh;

    if (p.check_info && p.status[kInfo] != 0) return;  // uniform: an earlier singular pivot

    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) & ~uintptr_t(1023));
    const int tiles_m = (p.M + TBM - 1) / TBM;
    const int tiles_n = (p.N + TBN - 1) / TBN;
    constexpr int kGroup = 8;
    const int bid = blockIdx.x;
    const int group = bid / (kGroup * tiles_n);
    const int first_m = group * kGroup;
    const int gsize = min(tiles_m - first_m, kGroup);
    const int in_group = bid % (kGroup * tiles_n);
    const int tm = first_m + in_group % gsize;
    const int tn = in_group / gsize;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int KT = (p.K + TBK - 1) / TBK;

    if (warp == 5) {
        tmem_alloc(&tmem_base_sh, TBN);
        tmem_relinquish();
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        mbar_init(&acc_bar, 1);
        fence_barrier_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_sh;
    bool ok = true;

    if (warp == 4) {
        if (lane == 0) {
            tma_prefetch_desc(&tmAh);
            tma_prefetch_desc(&tmBh);
            for (int kt = 0; kt < KT; ++kt) {
                const int s = kt % STAGES;
                const uint32_t ph = (kt / STAGES) & 1;
                if (!mbar_wait(&empty_bar[s], ph ^ 1, &p.status[kTimeout], 301)) { ok = false; break; }
                uint8_t* st = smem + s * kStage;
                mbar_arrive_expect_tx(&full_bar[s], kStage);
                const int ka = p.a_x0 + kt * TBK, kb = p.b_x0 + kt * TBK;
                tma_load_2d(st, &tmAh, ka, p.a_y0 + tm * TBM, &full_bar[s]);
                tma_load_2d(st + kTileB, &tmBh, kb, p.b_y0 + tn * TBN, &full_bar[s]);
                if (SPLIT == 3) {
                    tma_load_2d(st + 2 * kTileB, &tmAl, ka, p.a_y0 + tm * TBM, &full_bar[s]);
                    tma_load_2d(st + 3 * kTileB, &tmBl, kb, p.b_y0 + tn * TBN, &full_bar[s]);
                }
            }
        }
    } else if (warp == 5) {
        if (lane == 0) {
            constexpr uint32_t idesc = tf32_idesc();
            for (int kt = 0; kt < KT; ++kt) {
                const int s = kt % STAGES;
                const uint32_t ph = (kt / STAGES) & 1;
                if (!mbar_wait(&full_bar[s], ph, &p.status[kTimeout], 302)) { ok = false; break; }
                tc_fence_after();
                const uint32_t sa = smem_u32(smem + s * kStage);
#pragma unroll
                for (int kk = 0; kk < TBK / 8; ++kk) {
                    const uint32_t off = kk * 32;  // 8 tf32 values = 32 bytes along K inside the swizzle row
                    const uint64_t ah = sw128_desc(sa + off), bh = sw128_desc(sa + kTileB + off);
                    const uint32_t acc = (kt > 0 || kk > 0) ? 1u : 0u;
                    umma_tf32(tmem, ah, bh, idesc, acc);
                    if (SPLIT == 3) {
                        const uint64_t al = sw128_desc(sa + 2 * kTileB + off), bl = sw128_desc(sa + 3 * kTileB + off);
                        umma_tf32(tmem, ah, bl, idesc, 1u);
                        umma_tf32(tmem, al, bh, idesc, 1u);
                    }
                }
                umma_commit(&empty_bar[s]);  // frees the stage when these MMAs have read it
            }
            umma_commit(&acc_bar);  // accumulator complete
        }
    } else {
        // epilogue warps 0-3: TMEM lanes 32w..32w+31 = tile rows.  Column group cg (32 columns) of
        // row r goes to staging tile cg, 128-byte row r, 16-byte chunk j at position j ^ (r & 7).
        if (mbar_wait(&acc_bar, 0, &p.status[kTimeout], 303)) {
            tc_fence_after();
            const int r = warp * 32 + lane;
            const float sgn = p.op == B2M_DO_SUB ? -1.0f : 1.0f;
#pragma unroll 1
            for (int cg = 0; cg < TBN / 32; ++cg) {
                uint32_t v[32];
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cg * 32), *reinterpret_cast<uint32_t(*)[16]>(v));
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cg * 32 + 16),
                          *reinterpret_cast<uint32_t(*)[16]>(v + 16));
                uint8_t* tile = smem + cg * (TBM * 128);
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const float4 f = make_float4(sgn * __uint_as_float(v[4 * j]), sgn * __uint_as_float(v[4 * j + 1]),
                                                 sgn * __uint_as_float(v[4 * j + 2]), sgn * __uint_as_float(v[4 * j + 3]));
                    *reinterpret_cast<float4*>(tile + r * 128 + ((j ^ (r & 7)) << 4)) = f;
                }
            }
            fence_proxy_async();
            asm volatile("bar.sync 1, 128;\n" ::: "memory");  // the four epilogue warps
            if (threadIdx.x == 0) {
                for (int cg = 0; cg < TBN / 32; ++cg) {
                    const int x = p.c_x0 + tn * TBN + cg * 32, y = p.c_y0 + tm * TBM;
                    if (tn * TBN + cg * 32 >= p.N) break;
                    const uint32_t src = smem_u32(smem + cg * (TBM * 128));
                    if (p.op == B2M_DO_NONE)
                        asm volatile(
                            "cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];\n" ::"l"(
                                reinterpret_cast<uint64_t>(&tmC)),
                            "r"(x), "r"(y), "r"(src)
                            : "memory");
                    else
                        asm volatile(
                            "cp.reduce.async.bulk.tensor.2d.global.shared::cta.add.tile.bulk_group [%0, {%1, %2}], "
                            "[%3];\n" ::"l"(reinterpret_cast<uint64_t>(&tmC)),
                            "r"(x), "r"(y), "r"(src)
                            : "memory");
                }
                asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
                asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
            }
        }
    }
    (void)ok;
    tc_fence_before();
    __syncthreads();
    if (warp == 5) {
        tc_fence_after();
        tmem_dealloc(tmem, TBN);
    }
}

// hi = x with the 13 low mantissa bits cleared (exact in TF32), lo = x - hi (exact in FP32).
// Reads src (rows x cols, row stride lds); writes hi / lo (optionally transposed: out[c][r]).
__global__ void tf32_split_kernel(const float* __restrict__ src, int64_t lds, int rows, int cols, float* hi, float* lo,
                                  int64_t ldo, int transpose) {
    __shared__ float tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    for (int i = ty; i < 32; i += 8) {
        const int r = by + i, c = bx + tx;
        tile[i][tx] = (r < rows && c < cols) ? src[(int64_t)r * lds + c] : 0.f;
    }
    __syncthreads();
    for (int i = ty; i < 32; i += 8) {
        float x;
        int orow, ocol;
        if (transpose) {
            x = tile[tx][i];
            orow = bx + i;
            ocol = by + tx;
            if (orow >= cols || ocol >= rows) continue;
        } else {
            x = tile[i][tx];
            orow = by + i;
            ocol = bx + tx;
            if (orow >= rows || ocol >= cols) continue;
        }
        const float h = __uint_as_float(__float_as_uint(x) & 0xFFFFE000u);
        hi[(int64_t)orow * ldo + ocol] = h;
        if (lo) lo[(int64_t)orow * ldo + ocol] = x - h;
    }
}

template <int SPLIT>
int32_t launch_tc(Ctx* ctx, cudaStream_t st, const CUtensorMap* maps, const TcArgs& a) {
    constexpr int NOPS = SPLIT == 3 ? 4 : 2;
    constexpr int STAGES = SPLIT == 3 ? 3 : 5;
    constexpr int smem = STAGES * NOPS * kTileB + 1024;
    static_assert(STAGES * NOPS * kTileB >= (TBN / 32) * TBM * 128, "epilogue staging must fit in the stages");
    std::atomic<int>& attr = device_flag((const void*)sgemm_tc_kernel<SPLIT>, 0, ctx->device);
    if (!attr.load()) {
        B2M_CU(ctx, cudaFuncSetAttribute(sgemm_tc_kernel<SPLIT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        // the largest carveout, so that an SM running a tile still has shared memory for the
        // (small) panel kernels of the LU that may run beside this GEMM
        B2M_CU(ctx, cudaFuncSetAttribute(sgemm_tc_kernel<SPLIT>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         (int)cudaSharedmemCarveoutMaxShared));
        attr.store(1);
    }
    const int tiles = (int)(ceil_div(a.M, TBM) * ceil_div(a.N, TBN));
    prof_begin(ctx, st, kClsTcGemm);
    B2M_CU(ctx, launch_k(ctx, sgemm_tc_kernel<SPLIT>, dim3(tiles), dim3(kTcThreads), smem, st, maps[0], maps[1],
                         maps[2], maps[3], maps[4], a));
    prof_end(ctx, st, kClsTcGemm, 2.0 * a.M * a.N * a.K * SPLIT);
    B2M_LAUNCHED(ctx);
    return B2M_OK;
}

}  // namespace

int32_t tf32_split(Ctx* ctx, cudaStream_t st, const float* src, int64_t lds, int64_t rows, int64_t cols, float* hi,
                   float* lo, int64_t ldo, bool transpose) {
    if (rows <= 0 || cols <= 0) return B2M_OK;
    dim3 grid((unsigned)ceil_div(cols, 32), (unsigned)ceil_div(rows, 32));
    tf32_split_kernel<<<grid, dim3(32, 8), 0, st>>>(src, lds, (int)rows, (int)cols, hi, lo, ldo, transpose ? 1 : 0);
    B2M_LAUNCHED(ctx);
    return B2M_OK;
}

int32_t sgemm_tc(Ctx* ctx, cudaStream_t st, const FOperand& Ah, const float* Al_base, const FOperand& Bh,
                 const float* Bl_base, float* C, int64_t ldc, int64_t M, int64_t N, int64_t K, int op, int split,
                 bool check_info) {
    if (M <= 0 || N <= 0) return B2M_OK;
    if (K <= 0) {
        if (op == B2M_DO_NONE) B2M_CU(ctx, cudaMemset2DAsync(C, ldc * 4, 0, N * 4, M, st));
        return B2M_OK;
    }
    if ((Ah.c0 & 3) || (Bh.c0 & 3) || (Ah.ld & 3) || (Bh.ld & 3))
        return fail(ctx, B2M_ERR_DIM, "sgemm_tc: TMA origins/strides must be multiples of 4 floats");
    if (split == 3 && (!Al_base || !Bl_base)) return fail(ctx, B2M_ERR_ARG, "sgemm_tc: 3xTF32 needs lo operands");
    if (!aligned16(C) || (ldc & 3)) return fail(ctx, B2M_ERR_DIM, "sgemm_tc: C must be 16-byte aligned, ldc % 4 == 0");
    CUtensorMap maps[5];
    B2M_TRY(encode_tmap_2d(ctx, &maps[4], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, C, N, M, ldc * 4, 32, TBM,
                           CU_TENSOR_MAP_SWIZZLE_128B));
    B2M_TRY(encode_tmap_2d(ctx, &maps[0], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, Ah.base, Ah.cols, Ah.rows, Ah.ld * 4,
                           TBK, TBM, CU_TENSOR_MAP_SWIZZLE_128B));
    B2M_TRY(encode_tmap_2d(ctx, &maps[2], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, Bh.base, Bh.cols, Bh.rows, Bh.ld * 4,
                           TBK, TBN, CU_TENSOR_MAP_SWIZZLE_128B));
    if (split == 3) {
        B2M_TRY(encode_tmap_2d(ctx, &maps[1], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, Al_base, Ah.cols, Ah.rows, Ah.ld * 4,
                               TBK, TBM, CU_TENSOR_MAP_SWIZZLE_128B));
        B2M_TRY(encode_tmap_2d(ctx, &maps[3], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, Bl_base, Bh.cols, Bh.rows, Bh.ld * 4,
                               TBK, TBN, CU_TENSOR_MAP_SWIZZLE_128B));
    } else {
        maps[1] = maps[0];
        maps[3] = maps[2];
    }
    TcArgs a;
    a.M = (int)M; a.N = (int)N; a.K = (int)K;
    a.c_x0 = 0; a.c_y0 = 0;
    a.a_x0 = (int)Ah.c0; a.a_y0 = (int)Ah.r0;
    a.b_x0 = (int)Bh.c0; a.b_y0 = (int)Bh.r0;
    a.C = C; a.ldc = ldc; a.op = op; a.split = split;
    a.status = ctx->d_status;
    a.check_info = check_info ? 1 : 0;
    return split == 3 ? launch_tc<3>(ctx, st, maps, a) : launch_tc<1>(ctx, st, maps, a);
}

}  // namespace b2m
