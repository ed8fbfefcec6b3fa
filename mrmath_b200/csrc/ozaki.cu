// ozaki.cu -- FP64 matrix product emulated on the INT8 tensor cores (Ozaki scheme, integer slices).
//
// There is no counterpart in the reference; it is an alternative engine for MatrixMult /
// MatrixMultEx (MatrixASMStubSwitch.pas:769-782) whose result is judged against the FP64 oracle.
//
//   * every row i of A is scaled by 2^-ea_i (ea_i: exponent of the row's largest magnitude) and
//     every column j of B by 2^-eb_j, so each scaled entry lies in (-1, 1);
//   * a scaled entry x is cut into s signed 7-bit slices: x = sum_p x_p 2^-7p with x_p = trunc of
//     the remaining fraction times 2^7, |x_p| <= 127 (exact for the top 7 s bits);
//   * C = 2^(ea_i + eb_j) sum_d 2^-7d S_d with S_d = sum_{p+q=d} A_p B_q over the pairs with
//     d <= s + 1 (the dropped pairs are below 2^-7(s+1) of the scaled products).  Every S_d is an
//     exact int32 sum (|A_p B_q| <= 127^2 K per pair; K is cut into chunks that keep s 127^2 K below
//     2^31), accumulated on tcgen05.mma kind::i8 in TMEM;
//   * ozaki_kmajor_kernel (s <= 8, the default s = 8): see its comment below; ozaki_gemm_kernel
//     (s = 9, 10): warp 8 issues the TMA loads of 128 x 128 int8 tiles (128-byte swizzle),
//     one thread of warp 9 issues 4 MMAs (K = 32) per tile pair into one of two 128-column TMEM
//     accumulators, and warps 0-7 drain each finished S_d into FP64 registers (warp w: TMEM lanes
//     32 (w % 4).., columns 64 (w / 4)..), scaling by 2^-7d, while the next S_d accumulates in the
//     other buffer.  The final FP64 tile is scaled by 2^(ea_i + eb_j) and stored (op none/add/sub).
#include <cfloat>

#include "common.cuh"
#include "kernels.cuh"

namespace b2m {
namespace {

constexpr int OBM = 128, OBN = 128, OBK = 128;   // tile, k-step in int8 elements (= bytes)
constexpr int kOzTile = OBM * OBK;               // 16 KiB per operand tile
constexpr int kOzStages = 6;
constexpr int kOzThreads = 320;                  // 8 epilogue warps, producer, MMA
constexpr int kOzMaxSlices = 10;

struct OzArgs {
    int M, N, K, s;
    int kchunk;            // k-steps per accumulation chunk
    const int32_t* ea;     // row exponents of A
    const int32_t* eb;     // column exponents of B
    double* C;
    int64_t ldc;
    int op;
    int32_t* status;
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
__device__ __forceinline__ void umma_i8(uint32_t tmem_c, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_c),
        "l"(da), "l"(db), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     smem_u32(bar))
                 : "memory");
}
// K-major operand tile, 128-byte swizzle: 128-byte rows, 8-row groups 1024 bytes apart
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}
// s8 x s8 -> s32, both K-major, M = 128, N = 128
__host__ __device__ constexpr uint32_t i8_idesc() {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(OBN >> 3) << 17) | ((uint32_t)(OBM >> 4) << 24);
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

__global__ void __launch_bounds__(kOzThreads, 1)
    ozaki_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, OzArgs p) {
    extern __shared__ uint8_t oz_smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[kOzStages];
    __shared__ __align__(8) uint64_t empty_bar[kOzStages];
    __shared__ __align__(8) uint64_t accf_bar[2];   // S_d complete in buffer b
    __shared__ __align__(8) uint64_t acce_bar[2];   // buffer b drained by the epilogue
    __shared__ uint32_t tmem_base_sh;

    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(oz_smem_raw) + 1023) & ~uintptr_t(1023));
    const int tiles_m = (p.M + OBM - 1) / OBM, tiles_n = (p.N + OBN - 1) / OBN;
    constexpr int kGroup = 8;
    const int bid = blockIdx.x;
    const int group = bid / (kGroup * tiles_n);
    const int first_m = group * kGroup;
    const int gsize = min(tiles_m - first_m, kGroup);
    const int in_group = bid % (kGroup * tiles_n);
    const int tm = first_m + in_group % gsize, tn = in_group / gsize;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int KT = (p.K + OBK - 1) / OBK;
    const int nchunks = (KT + p.kchunk - 1) / p.kchunk;
    const int s = p.s;

    if (warp == 9) {
        tmem_alloc(&tmem_base_sh, 2 * OBN);
        tmem_relinquish();
    }
    if (threadIdx.x == 0) {
        for (int i = 0; i < kOzStages; ++i) {
            mbar_init(&full_bar[i], 1);
            mbar_init(&empty_bar[i], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&accf_bar[b], 1);
            mbar_init(&acce_bar[b], 8);
        }
        fence_barrier_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_sh;
    int32_t* tmo = &p.status[kTimeout];

    if (warp == 8) {
        // producer: the same (chunk, d, p, k-step) schedule as the MMA issuer
        if (lane == 0) {
            tma_prefetch_desc(&tmA);
            tma_prefetch_desc(&tmB);
            int it = 0;
            bool ok = true;
            for (int ch = 0; ch < nchunks && ok; ++ch) {
                const int k0 = ch * p.kchunk, k1 = min(KT, k0 + p.kchunk);
                for (int d = 2; d <= s + 1 && ok; ++d)
                    for (int pa = max(1, d - s); pa <= min(s, d - 1) && ok; ++pa) {
                        const int pb = d - pa;
                        for (int kt = k0; kt < k1; ++kt, ++it) {
                            const int st = it % kOzStages;
                            if (!mbar_wait(&empty_bar[st], ((it / kOzStages) & 1) ^ 1, tmo, 401)) { ok = false; break; }
                            uint8_t* sp = smem + st * 2 * kOzTile;
                            mbar_arrive_expect_tx(&full_bar[st], 2 * kOzTile);
                            tma_load_2d(sp, &tmA, kt * OBK, (pa - 1) * p.M + tm * OBM, &full_bar[st]);
                            tma_load_2d(sp + kOzTile, &tmB, kt * OBK, (pb - 1) * p.N + tn * OBN, &full_bar[st]);
                        }
                    }
            }
        }
    } else if (warp == 9) {
        if (lane == 0) {
            constexpr uint32_t idesc = i8_idesc();
            int it = 0, unit = 0;
            bool ok = true;
            for (int ch = 0; ch < nchunks && ok; ++ch) {
                const int k0 = ch * p.kchunk, k1 = min(KT, k0 + p.kchunk);
                for (int d = 2; d <= s + 1 && ok; ++d, ++unit) {
                    const int b = unit & 1;
                    // the epilogue must have drained this buffer (unit - 2) before it is overwritten
                    if (unit >= 2 && !mbar_wait(&acce_bar[b], ((unit >> 1) - 1) & 1, tmo, 402)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t tacc = tmem + (uint32_t)(b * OBN);
                    bool first = true;
                    for (int pa = max(1, d - s); pa <= min(s, d - 1) && ok; ++pa) {
                        for (int kt = k0; kt < k1; ++kt, ++it) {
                            const int st = it % kOzStages;
                            if (!mbar_wait(&full_bar[st], (it / kOzStages) & 1, tmo, 403)) { ok = false; break; }
                            tc_fence_after();
                            const uint32_t sa = smem_u32(smem + st * 2 * kOzTile);
#pragma unroll
                            for (int kk = 0; kk < OBK / 32; ++kk) {
                                const uint32_t off = kk * 32;
                                umma_i8(tacc, sw128_desc(sa + off), sw128_desc(sa + kOzTile + off), idesc, first ? 0u : 1u);
                                first = false;
                            }
                            umma_commit(&empty_bar[st]);
                        }
                    }
                    umma_commit(&accf_bar[b]);
                }
            }
        }
    } else {
        // epilogue warps 0-7: rows 32 (warp % 4) + lane, columns 64 (warp / 4) .. + 63
        const int q = warp & 3, h = warp >> 2;
        double acc[64];
#pragma unroll
        for (int c = 0; c < 64; ++c) acc[c] = 0.0;
        int unit = 0;
        bool ok = true;
        for (int ch = 0; ch < nchunks && ok; ++ch) {
            for (int d = 2; d <= s + 1; ++d, ++unit) {
                const int b = unit & 1;
                if (!mbar_wait(&accf_bar[b], (unit >> 1) & 1, tmo, 404)) { ok = false; break; }
                tc_fence_after();
                const double sc = ldexp(1.0, -7 * d);
                const uint32_t ta = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * OBN + h * 64);
#pragma unroll
                for (int c0 = 0; c0 < 64; c0 += 16) {
                    uint32_t r[16];
                    tmem_ld16(ta + (uint32_t)c0, r);
#pragma unroll
                    for (int e = 0; e < 16; ++e) acc[c0 + e] = fma((double)(int32_t)r[e], sc, acc[c0 + e]);
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&acce_bar[b]);
            }
        }
        const int row = tm * OBM + q * 32 + lane;
        if (ok && row < p.M) {
            const double sa = ldexp(1.0, p.ea[row]);
            double* crow = p.C + (int64_t)row * p.ldc + tn * OBN + h * 64;
            const int cbase = tn * OBN + h * 64;
#pragma unroll
            for (int c = 0; c < 64; ++c) {
                const int col = cbase + c;
                if (col < p.N) {
                    const double v = acc[c] * sa * ldexp(1.0, p.eb[col]);
                    if (p.op == B2M_DO_NONE) crow[c] = v;
                    else if (p.op == B2M_DO_ADD) crow[c] += v;
                    else crow[c] -= v;
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 9) {
        tc_fence_after();
        tmem_dealloc(tmem, 2 * OBN);
    }
}

// ---- k-major variant (s <= 8 slices): every slice tile is loaded once per k-step and reused by
// every pair it belongs to.  A CTA computes a 128 x 64 tile of C with all s accumulators S_d
// (d = 2 .. s + 1, 64 TMEM columns each, 512 in all) live for the whole K range: per 32-wide
// k-step the producer (warp 8) loads the s slice tiles of A (128 x 32 bytes) and of B (64 x 32),
// 32-byte swizzle, into one of four stages; the MMA issuer (one thread of warp 9) runs the
// s (s + 1) / 2 pairs of the step (one K = 32 MMA each) into the accumulator of d = p + q; the
// epilogue warps drain the accumulators into FP64 once per K chunk (a chunk keeps every S_d an
// exact int32 sum).  Per k-step the tensor pipe gets s (s + 1) / 2 MMAs for 6 s KiB of operands,
// about three times the reuse of the pair-major kernel above, whose slice pairs each reload both
// tiles.
constexpr int KBM = 128, KBN = 64, KBK = 32;
constexpr int kKmTileA = KBM * KBK, kKmTileB = KBN * KBK;  // 4 KiB, 2 KiB
constexpr int kKmMaxSlices = 8;
constexpr int kKmStages = 4;  // 4 x 48 KiB: three stages in flight hide the TMA latency behind the MMAs

// K-major operand tile, 32-byte swizzle: 32-byte rows (one K = 32 MMA), 8-row groups 256 bytes apart
__device__ __forceinline__ uint64_t sw32_desc(uint32_t saddr) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(256 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)6 << 61);
}
__host__ __device__ constexpr uint32_t i8_idesc_m128n64() {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(KBN >> 3) << 17) | ((uint32_t)(KBM >> 4) << 24);
}

// the s (s + 1) / 2 MMAs of one k-step for a compile-time s: descriptors are the stage's base
// descriptors plus constants, and the first MMA of every accumulator (pa = 1 in this order) of a
// chunk's first k-step starts it
template <int S>
__device__ __forceinline__ void km_issue_step(uint32_t tmem, uint64_t da0, uint64_t db0, uint32_t idesc, bool first) {
#pragma unroll
    for (int pa = 1; pa <= S; ++pa) {
#pragma unroll
        for (int pb = 1; pa + pb <= S + 1; ++pb) {
            const int d = pa + pb;
            umma_i8(tmem + (uint32_t)((d - 2) * KBN), da0 + (uint64_t)(((pa - 1) * kKmTileA) >> 4),
                    db0 + (uint64_t)(((pb - 1) * kKmTileB) >> 4), idesc, (first && pa == 1) ? 0u : 1u);
        }
    }
}

__global__ void __launch_bounds__(kOzThreads, 1)
    ozaki_kmajor_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, OzArgs p) {
    extern __shared__ uint8_t km_smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[kKmStages];
    __shared__ __align__(8) uint64_t empty_bar[kKmStages];
    __shared__ __align__(8) uint64_t accf_bar;   // the chunk's accumulators are complete
    __shared__ __align__(8) uint64_t acce_bar;   // ... and drained by the epilogue
    __shared__ uint32_t tmem_base_sh;

    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(km_smem_raw) + 1023) & ~uintptr_t(1023));
    const int s = p.s;
    const int stage_bytes = s * (kKmTileA + kKmTileB);
    const int tiles_m = (p.M + KBM - 1) / KBM, tiles_n = (p.N + KBN - 1) / KBN;
    constexpr int kGroup = 8;
    const int bid = blockIdx.x;
    const int group = bid / (kGroup * tiles_n);
    const int first_m = group * kGroup;
    const int gsize = min(tiles_m - first_m, kGroup);
    const int in_group = bid % (kGroup * tiles_n);
    const int tm = first_m + in_group % gsize, tn = in_group / gsize;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int KT = (p.K + KBK - 1) / KBK;
    const int nchunks = (KT + p.kchunk - 1) / p.kchunk;

    if (warp == 9) {
        tmem_alloc(&tmem_base_sh, 512);
        tmem_relinquish();
    }
    if (threadIdx.x == 0) {
        for (int i = 0; i < kKmStages; ++i) {
            mbar_init(&full_bar[i], 1);
            mbar_init(&empty_bar[i], 1);
        }
        mbar_init(&accf_bar, 1);
        mbar_init(&acce_bar, 8);
        fence_barrier_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_sh;
    int32_t* tmo = &p.status[kTimeout];

    if (warp == 8) {
        if (lane == 0) {
            tma_prefetch_desc(&tmA);
            tma_prefetch_desc(&tmB);
            bool ok = true;
            for (int kt = 0; kt < KT && ok; ++kt) {
                const int st = kt % kKmStages;
                if (!mbar_wait(&empty_bar[st], ((kt / kKmStages) & 1) ^ 1, tmo, 411)) { ok = false; break; }
                uint8_t* sp = smem + st * stage_bytes;
                mbar_arrive_expect_tx(&full_bar[st], stage_bytes);
                for (int q = 0; q < s; ++q) {
                    tma_load_2d(sp + q * kKmTileA, &tmA, kt * KBK, q * p.M + tm * KBM, &full_bar[st]);
                    tma_load_2d(sp + s * kKmTileA + q * kKmTileB, &tmB, kt * KBK, q * p.N + tn * KBN, &full_bar[st]);
                }
            }
        }
    } else if (warp == 9) {
        if (lane == 0) {
            constexpr uint32_t idesc = i8_idesc_m128n64();
            bool ok = true;
            for (int ch = 0; ch < nchunks && ok; ++ch) {
                const int k0 = ch * p.kchunk, k1 = min(KT, k0 + p.kchunk);
                // the epilogue must have drained the previous chunk before the accumulators restart
                if (ch > 0 && !mbar_wait(&acce_bar, (ch - 1) & 1, tmo, 412)) { ok = false; break; }
                tc_fence_after();
                uint32_t started = 0u;  // accumulators written in this chunk (bit d - 2)
                for (int kt = k0; kt < k1; ++kt) {
                    const int st = kt % kKmStages;
                    if (!mbar_wait(&full_bar[st], (kt / kKmStages) & 1, tmo, 413)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t sa = smem_u32(smem + st * stage_bytes);
                    const uint32_t sb = sa + (uint32_t)(s * kKmTileA);
                    if (s == kKmMaxSlices) {
                        km_issue_step<kKmMaxSlices>(tmem, sw32_desc(sa), sw32_desc(sb), idesc, kt == k0);
                    } else {
                        for (int pa = 1; pa <= s; ++pa) {
                            for (int pb = 1; pa + pb <= s + 1; ++pb) {
                                const int d = pa + pb;
                                const uint32_t tacc = tmem + (uint32_t)((d - 2) * KBN);
                                const uint32_t acc = (started >> (d - 2)) & 1u;
                                umma_i8(tacc, sw32_desc(sa + (uint32_t)((pa - 1) * kKmTileA)),
                                        sw32_desc(sb + (uint32_t)((pb - 1) * kKmTileB)), idesc, acc);
                                started |= 1u << (d - 2);
                            }
                        }
                    }
                    umma_commit(&empty_bar[st]);
                }
                umma_commit(&accf_bar);
            }
        }
    } else {
        // epilogue warps 0-7: rows 32 (warp % 4) + lane, columns 32 (warp / 4) .. + 31
        const int q4 = warp & 3, h = warp >> 2;
        double acc[32];
#pragma unroll
        for (int c = 0; c < 32; ++c) acc[c] = 0.0;
        bool ok = true;
        for (int ch = 0; ch < nchunks && ok; ++ch) {
            if (!mbar_wait(&accf_bar, ch & 1, tmo, 414)) { ok = false; break; }
            tc_fence_after();
            for (int d = 2; d <= s + 1; ++d) {
                const double sc = ldexp(1.0, -7 * d);
                const uint32_t ta = tmem + ((uint32_t)(q4 * 32) << 16) + (uint32_t)((d - 2) * KBN + h * 32);
#pragma unroll
                for (int c0 = 0; c0 < 32; c0 += 16) {
                    uint32_t r[16];
                    tmem_ld16(ta + (uint32_t)c0, r);
#pragma unroll
                    for (int e = 0; e < 16; ++e) acc[c0 + e] = fma((double)(int32_t)r[e], sc, acc[c0 + e]);
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acce_bar);
        }
        const int row = tm * KBM + q4 * 32 + lane;
        if (ok && row < p.M) {
            const double sa = ldexp(1.0, p.ea[row]);
            double* crow = p.C + (int64_t)row * p.ldc + tn * KBN + h * 32;
            const int cbase = tn * KBN + h * 32;
#pragma unroll
            for (int c = 0; c < 32; ++c) {
                const int col = cbase + c;
                if (col < p.N) {
                    const double v = acc[c] * sa * ldexp(1.0, p.eb[col]);
                    if (p.op == B2M_DO_NONE) crow[c] = v;
                    else if (p.op == B2M_DO_ADD) crow[c] += v;
                    else crow[c] -= v;
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 9) {
        tc_fence_after();
        tmem_dealloc(tmem, 512);
    }
}

// exponent e with max|x| * 2^-e < 1 (0 for an all-zero row/column)
__device__ __forceinline__ int exp_of(double m) {
    if (!(m > 0.0)) return 0;
    int e;
    frexp(m, &e);
    return e;
}

// row exponents of A (M x K, row stride lda): one warp per row
__global__ void ozaki_row_exp_kernel(const double* A, int64_t lda, int M, int K, int32_t* ea) {
    const int row = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (row >= M) return;
    double m = 0.0;
    for (int k = lane; k < K; k += 32) m = fmax(m, fabs(A[(int64_t)row * lda + k]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) ea[row] = exp_of(m);
}

// column exponents of B (K x N, row stride ldb): a thread per column
__global__ void ozaki_col_exp_kernel(const double* B, int64_t ldb, int K, int N, int32_t* eb) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= N) return;
    double m = 0.0;
    for (int k = 0; k < K; ++k) m = fmax(m, fabs(B[(int64_t)k * ldb + col]));
    eb[col] = exp_of(m);
}

// A slices: A8[p][i][k] (p < s, row stride Kp bytes)
__global__ void ozaki_slice_a_kernel(const double* A, int64_t lda, int M, int K, const int32_t* ea, int s,
                                     int8_t* A8, int64_t Kp) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)M * Kp) return;
    const int i = (int)(e / Kp), k = (int)(e - (int64_t)i * Kp);
    double x = k < K ? A[(int64_t)i * lda + k] * ldexp(1.0, -ea[i]) : 0.0;
    for (int p = 0; p < s; ++p) {
        x *= 128.0;
        const double v = trunc(x);
        x -= v;
        A8[((int64_t)p * M + i) * Kp + k] = (int8_t)v;
    }
}

// B slices, transposed to K-major: B8[q][j][k] (row stride Kp bytes); 32 x 32 tiles through
// shared memory so that both the read (along j) and the write (along k) are coalesced
__global__ void ozaki_slice_b_kernel(const double* B, int64_t ldb, int K, int N, const int32_t* eb, int s,
                                     int8_t* B8, int64_t Kp) {
    __shared__ double tile[32][33];
    const int k0 = blockIdx.y * 32, j0 = blockIdx.x * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    for (int r = ty; r < 32; r += 8) {
        const int k = k0 + r, j = j0 + tx;
        tile[r][tx] = (k < K && j < N) ? B[(int64_t)k * ldb + j] * ldexp(1.0, -eb[j]) : 0.0;
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) {
        const int j = j0 + r, k = k0 + tx;
        if (j >= N || k >= Kp) continue;
        double x = tile[tx][r];
        for (int q = 0; q < s; ++q) {
            x *= 128.0;
            const double v = trunc(x);
            x -= v;
            B8[((int64_t)q * N + j) * Kp + k] = (int8_t)v;
        }
    }
}

}  // namespace

// C (M x N, ldc) op= A (M x K, lda) * B (K x N, ldb), all FP64 device memory, on the INT8 tensor
// cores with s slices per operand.
int32_t ozaki_gemm(Ctx* ctx, cudaStream_t st, const double* A, int64_t lda, const double* B, int64_t ldb, double* C,
                   int64_t ldc, int64_t M, int64_t N, int64_t K, int op, int s) {
    if (M <= 0 || N <= 0) return B2M_OK;
    if (s < 2 || s > kOzMaxSlices) return fail(ctx, B2M_ERR_ARG, "ozaki: slices must be in [2, %d]", kOzMaxSlices);
    if (M > (1 << 28) / kOzMaxSlices || N > (1 << 28) / kOzMaxSlices || K > (1 << 30))
        return fail(ctx, B2M_ERR_UNSUPPORTED, "ozaki: operand too large");
    if (K <= 0) {
        if (op == B2M_DO_NONE) B2M_CU(ctx, cudaMemset2DAsync(C, ldc * 8, 0, N * 8, M, st));
        return B2M_OK;
    }
    const int64_t Kp = round_up(K, 128);
    // exact int32 accumulation: s pairs of |127 * 127| products over one chunk
    const int64_t kchunk_elems = ((int64_t)2147483647 / ((int64_t)s * 127 * 127)) / OBK * OBK;
    const int kchunk = (int)std::max<int64_t>(1, kchunk_elems / OBK);
    void *pe, *pa, *pb;
    B2M_TRY(ws_get(ctx, kWsSmall, (size_t)(M + N) * 4 + 256, &pe));
    B2M_TRY(ws_get(ctx, kWsMatD, (size_t)s * M * Kp, &pa));
    B2M_TRY(ws_get(ctx, kWsH, (size_t)s * N * Kp, &pb));
    int32_t* ea = (int32_t*)pe;
    int32_t* eb = ea + M;
    int8_t* A8 = (int8_t*)pa;
    int8_t* B8 = (int8_t*)pb;
    ozaki_row_exp_kernel<<<(unsigned)ceil_div(M, 8), 256, 0, st>>>(A, lda, (int)M, (int)K, ea);
    B2M_LAUNCHED(ctx);
    ozaki_col_exp_kernel<<<(unsigned)ceil_div(N, 256), 256, 0, st>>>(B, ldb, (int)K, (int)N, eb);
    B2M_LAUNCHED(ctx);
    prof_begin(ctx, st, kClsOther);
    ozaki_slice_a_kernel<<<(unsigned)ceil_div(M * Kp, 256), 256, 0, st>>>(A, lda, (int)M, (int)K, ea, s, A8, Kp);
    dim3 gb((unsigned)ceil_div(N, 32), (unsigned)ceil_div(Kp, 32));
    ozaki_slice_b_kernel<<<gb, dim3(32, 8), 0, st>>>(B, ldb, (int)K, (int)N, eb, s, B8, Kp);
    prof_end(ctx, st, kClsOther, 8.0 * (M * K + K * N) + (double)s * Kp * (M + N));  // bytes
    B2M_LAUNCHED(ctx);
    CUtensorMap ma, mb;
    if (s <= kKmMaxSlices) {
        // k-major kernel: all s accumulators in TMEM, K chunks that keep each S_d an exact int32 sum
        const int64_t kc_elems = ((int64_t)2147483647 / ((int64_t)s * 127 * 127)) / KBK * KBK;
        const int kc = (int)std::max<int64_t>(1, kc_elems / KBK);
        B2M_TRY(encode_tmap_2d(ctx, &ma, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, A8, (uint64_t)K, (uint64_t)s * M,
                               (uint64_t)Kp, KBK, KBM, CU_TENSOR_MAP_SWIZZLE_32B));
        B2M_TRY(encode_tmap_2d(ctx, &mb, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, B8, (uint64_t)K, (uint64_t)s * N,
                               (uint64_t)Kp, KBK, KBN, CU_TENSOR_MAP_SWIZZLE_32B));
        // the full-size request for every s: one CTA per SM, so that no second CTA waits for TMEM
        const int ksmem = kKmStages * kKmMaxSlices * (kKmTileA + kKmTileB) + 1024;
        std::atomic<int>& kattr = device_flag((const void*)ozaki_kmajor_kernel, 0, ctx->device);
        if (!kattr.load()) {
            B2M_CU(ctx, cudaFuncSetAttribute(ozaki_kmajor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, ksmem));
            kattr.store(1);
        }
        OzArgs ka{(int)M, (int)N, (int)K, s, kc, ea, eb, C, ldc, op, ctx->d_status};
        const int ktiles = (int)(ceil_div(M, KBM) * ceil_div(N, KBN));
        const double kpairs = (double)s * (s + 1) / 2.0;
        prof_begin(ctx, st, kClsTcGemm);
        ozaki_kmajor_kernel<<<ktiles, kOzThreads, ksmem, st>>>(ma, mb, ka);
        prof_end(ctx, st, kClsTcGemm, 2.0 * M * N * Kp * kpairs);  // int8 MMA operations
        B2M_LAUNCHED(ctx);
        return B2M_OK;
    }
    B2M_TRY(encode_tmap_2d(ctx, &ma, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, A8, (uint64_t)K, (uint64_t)s * M, (uint64_t)Kp,
                           OBK, OBM, CU_TENSOR_MAP_SWIZZLE_128B));
    B2M_TRY(encode_tmap_2d(ctx, &mb, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, B8, (uint64_t)K, (uint64_t)s * N, (uint64_t)Kp,
                           OBK, OBN, CU_TENSOR_MAP_SWIZZLE_128B));
    constexpr int smem = kOzStages * 2 * kOzTile + 1024;
    std::atomic<int>& attr = device_flag((const void*)ozaki_gemm_kernel, 0, ctx->device);
    if (!attr.load()) {
        B2M_CU(ctx, cudaFuncSetAttribute(ozaki_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        attr.store(1);
    }
    OzArgs a{(int)M, (int)N, (int)K, s, kchunk, ea, eb, C, ldc, op, ctx->d_status};
    const int tiles = (int)(ceil_div(M, OBM) * ceil_div(N, OBN));
    const double pairs = (double)s * (s + 1) / 2.0;
    prof_begin(ctx, st, kClsTcGemm);
    ozaki_gemm_kernel<<<tiles, kOzThreads, smem, st>>>(ma, mb, a);
    prof_end(ctx, st, kClsTcGemm, 2.0 * M * N * Kp * pairs);  // int8 MMA operations
    B2M_LAUNCHED(ctx);
    return B2M_OK;
}

}  // namespace b2m
