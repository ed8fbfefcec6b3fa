// lu_f32.cu -- FP32 LU factorisation for the mixed-precision solve.
//
// This factorisation only has to be good enough for iterative refinement to converge (the answer
// is judged by its FP64 backward error), so it is free to pick its pivots differently from the
// reference's FP64 LU.  It uses tournament pivoting (communication-avoiding LU, Grigori, Demmel
// and Xiang 2011), which removes the per-column grid-wide reduction that bounds a classic panel:
//
//   * outer panels of kNB = 256 columns, blocked right-looking: after a panel is factored, its
//     net row permutation is applied to the columns outside it (panel_permute_kernel), the rows
//     above the trailing matrix are solved with the panel's unit-lower block (U12, through the
//     leaves' L11^-1) and the trailing matrix is updated by tcgen05 GEMMs (TF32 or 3xTF32,
//     K = 256): the next panel's columns first, the rest on a side stream under the next panel's
//     leaves (look-ahead);
//   * inside a panel, 32-column leaves.  tslu_select_kernel runs Gaussian elimination with
//     partial pivoting on 512-row chunks in parallel; each chunk nominates 32 candidate rows, and
//     the last CTA of every group of 16 chunks (found with an atomic counter, no spinning) runs
//     the same elimination on the stacked candidates' original rows, up to a single root.  The
//     root's pivots are the leaf's pivots and its eliminated rows are the leaf's L11\U11;
//   * tslu_apply_kernel moves the chosen rows into place (a side buffer holds the rows whose
//     slots get overwritten, so the move is race free), forms L21 = A21 U11^-1 and applies the
//     leaf's rank-32 update to the rest of the panel; it records the moves in `perm` and in the
//     panel's row map, which the panel permutation applies to the other columns.
//
// The permutation is tracked in `perm` (row i of the factors is original row perm[i]); no LAPACK
// style interchange vector is produced because nothing downstream of the mixed solve needs one.
// A pivot whose magnitude is <= 10/FLT_MAX at the root sets status[kInfo] (the driver then
// falls back to the plain FP64 factorisation).
#include <cfloat>

#include "common.cuh"
#include "kernels.cuh"

namespace b2m {
namespace {

constexpr int kTsThreads = 256;
constexpr int kTsRpt = 2;                         // rows per thread in the elimination
constexpr int kTsRows = kTsThreads * kTsRpt;      // rows per chunk / per merge
constexpr int kTsFan = kTsRows / 32;              // candidate sets merged per tree node (16)
constexpr int kTsLevels = 4;
constexpr int kTsMaxCand = 2048;                  // nodes per level (rows <= 1M)
constexpr int kNB = 256;                          // outer panel width
constexpr int kApRows = 16;                       // rows per apply CTA

struct TsArgs {
    const float* A;
    int64_t ld;
    int n, lc0, w, oc0, pw;
    int* cand;            // [kTsLevels][kTsMaxCand][32] candidate row ids
    unsigned* counters;   // [kTsLevels][kTsMaxCand] arrival counters (zero between launches)
    float* top;           // [32][kNB]: final content of the leaf's top rows over the outer panel
    float* mvals;         // [32][kNB]: original content of the top rows that move below the leaf
    float* wmat;          // [32][kNB]: U11^-1 in the leaf's columns, U11^-1 U12 right of them
    int* moves;           // [0] moves, [1] moves below the top block, [2..66) dst, [66..130) src
    float* lmul;          // [32][kTsRows] the root elimination's multipliers
    int32_t* pmap;        // first leaf of a panel: pmap[i] = i for the panel's rows (identity)
    float* lpinv;         // [kNB / 32][32][32]: L11^-1 of each leaf of the outer panel
    int32_t* status;
};

// reciprocal: hardware approximation refined by one Newton step (a correctly rounded division
// costs ~300 cycles of dependent latency, and this factorisation only has to feed refinement)
__device__ __forceinline__ float rcp_nr(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r * fmaf(-x, r, 2.0f);
}

// Gaussian elimination with partial pivoting of up to 512 stacked rows (thread t holds stack rows
// t and t + 256 in registers) over w <= 32 columns.  Chooses w pivot rows (largest magnitude);
// s_win[j] = row id of pivot j and s_loc[j] = its stack index (-1 if the stack ran out).
//
// One column per iteration of a runtime loop (a compact body: unrolled multi-column steps spill
// out of the instruction cache).  Register indices stay compile-time because every row shifts
// left by one as its column is eliminated (the update writes v[k - 1]), so the current column is
// always v[0].  One barrier per column: before it, every warp's best lane publishes its candidate
// row, the reciprocal of its pivot value (computed by every lane while the warp reduction runs,
// so it is off the chain) and its stack slot (double-buffered by column parity), and folds its key
// into a shared maximum (atomicMax on the magnitude's bit pattern with the warp in the low 3 bits,
// so the lowest warp wins among magnitudes that agree to 2^-20); after it, every thread reads the
// maximum and then the winning row directly, with no further reduction.  The maximum words rotate
// through three slots: thread 0 clears the one of column j + 2 after the barrier of column j, when
// every read of it (column j - 1) is done and before any write (column j + 2).  For the root (lm
// given) the winner of column j is copied to s_u[j] (row j of U, from column j on) and every row's
// multiplier of column j goes to lm[j][stack index] (global scratch), which gives the rows of L;
// keeping them out of shared memory lets the CTA share an SM with a tensor-core GEMM.
struct GeppSmem {
    float4 cand[2][kTsThreads / 32][9];  // candidate rows by column parity and warp (column j first),
                                         // then (reciprocal of the pivot, stack slot, -, -)
    unsigned best[3];                    // packed maximum key of columns j, j + 1, j + 2 (mod 3)
    float4 u[32][8];                     // root: pivot rows as chosen
};

__device__ __forceinline__ void block_gepp(float (&v)[kTsRpt][32], const int (&rid)[kTsRpt], int w, int* s_win,
                                           int* s_loc, GeppSmem& g, float* lm) {
    static_assert(kTsThreads / 32 <= 8, "the warp index must fit the key's low 3 bits");
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    bool live[kTsRpt];
#pragma unroll
    for (int r = 0; r < kTsRpt; ++r) live[r] = rid[r] >= 0;
    if (t < 32) { s_win[t] = -1; s_loc[t] = -1; }
    if (t < 3) g.best[t] = 0u;
    __syncthreads();
    int b3 = 0;
#pragma unroll 1
    for (int j = 0; j < w; ++j) {
        const int b = j & 1;
        unsigned key = 0u;
        int rbest = 0;
#pragma unroll
        for (int r = 0; r < kTsRpt; ++r) {
            const unsigned k = live[r] ? __float_as_uint(fabsf(v[r][0])) + 1u : 0u;
            if (k > key) { key = k; rbest = r; }
        }
        float vsel = v[0][0];
#pragma unroll
        for (int r = 1; r < kTsRpt; ++r) vsel = rbest == r ? v[r][0] : vsel;
        const float rc = key > 1u ? rcp_nr(vsel) : 0.0f;  // a zero column eliminates nothing
        const unsigned wk = __reduce_max_sync(0xffffffffu, key);
        const unsigned bal = __ballot_sync(0xffffffffu, key == wk && key != 0u);
        if (wk != 0u && lane == __ffs(bal) - 1) {
#pragma unroll
            for (int r = 0; r < kTsRpt; ++r) {
                if (r == rbest) {
#pragma unroll
                    for (int q = 0; q < 8; ++q)
                        g.cand[b][warp][q] = make_float4(v[r][4 * q], v[r][4 * q + 1], v[r][4 * q + 2], v[r][4 * q + 3]);
                }
            }
            g.cand[b][warp][8] = make_float4(rc, __uint_as_float((unsigned)(rbest * kTsThreads + t)), 0.f, 0.f);
            atomicMax(&g.best[b3], ((wk > 8u ? wk : 8u) & ~7u) | (unsigned)(7 - warp));
        }
        __syncthreads();
        const unsigned pk = g.best[b3];
        if (t == 0) g.best[b3 == 0 ? 2 : b3 - 1] = 0u;  // the slot of column j + 2
        b3 = b3 == 2 ? 0 : b3 + 1;
        if (pk == 0u) break;  // no live row left anywhere (uniform)
        const int pwarp = 7 - (int)(pk & 7u);
        float pr[32];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const float4 f = g.cand[b][pwarp][q];
            pr[4 * q] = f.x; pr[4 * q + 1] = f.y; pr[4 * q + 2] = f.z; pr[4 * q + 3] = f.w;
        }
        const float4 meta = g.cand[b][pwarp][8];
        const float rcp = meta.x;
        const unsigned ps = __float_as_uint(meta.y);
        if (lm && t < 8) g.u[j][t] = g.cand[b][pwarp][t];
#pragma unroll
        for (int r = 0; r < kTsRpt; ++r) {
            if (ps == (unsigned)(r * kTsThreads + t)) {
                live[r] = false;
                s_win[j] = rid[r];
                s_loc[j] = r * kTsThreads + t;
            }
            const float l = live[r] ? v[r][0] * rcp : 0.f;
            if (lm) lm[j * kTsRows + r * kTsThreads + t] = l;
#pragma unroll
            for (int k = 1; k < 32; ++k) v[r][k - 1] = fmaf(-l, pr[k], v[r][k]);
            v[r][31] = 0.f;
        }
    }
    __syncthreads();
}

// loads columns [c0, c0 + w) of row `row` (zeros past w); rows are 128-byte aligned
__device__ __forceinline__ void load_leaf_row(const float* A, int64_t ld, int row, int c0, int w, float (&x)[32]) {
    if (row < 0) {
#pragma unroll
        for (int k = 0; k < 32; ++k) x[k] = 0.f;
        return;
    }
    const float4* p = reinterpret_cast<const float4*>(A + (int64_t)row * ld + c0);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const float4 f = __ldg(p + q);
        x[4 * q + 0] = f.x; x[4 * q + 1] = f.y; x[4 * q + 2] = f.z; x[4 * q + 3] = f.w;
    }
#pragma unroll
    for (int k = 0; k < 32; ++k)
        if (k >= w) x[k] = 0.f;
}

__global__ void __launch_bounds__(kTsThreads) tslu_select_kernel(TsArgs a) {
    __shared__ __align__(16) GeppSmem s_g;
    __shared__ int s_win[32], s_loc[32];
    __shared__ float s_lu[32][33];
    __shared__ __align__(16) float s_lt[32][32];  // s_lt[j][k] = L(k, j) for k > j, else 0
    __shared__ __align__(16) float s_ut[32][32];  // s_ut[i][k] = U(k, i) for k < i, else 0
    __shared__ float s_rdiag[32];
    __shared__ int s_last, s_bad;
    __shared__ int s_flag[32], s_outpos[32], s_mdst[64], s_msrc[64], s_nm, s_nout;
    if (a.status[kInfo] != 0) return;
    const int t = threadIdx.x;
    const int m = a.n - a.lc0;
    float v[kTsRpt][32];
    int rid[kTsRpt];
#pragma unroll
    for (int r = 0; r < kTsRpt; ++r) {
        const int row = a.lc0 + blockIdx.x * kTsRows + r * kTsThreads + t;
        rid[r] = row < a.n ? row : -1;
        load_leaf_row(a.A, a.ld, rid[r], a.lc0, a.w, v[r]);
        if (a.pmap && row < a.n) a.pmap[row] = row;
    }
    int node = blockIdx.x, count = (int)ceil_div(m, kTsRows), level = 0;
    for (;;) {
        block_gepp(v, rid, a.w, s_win, s_loc, s_g, count == 1 ? a.lmul : nullptr);
        if (count == 1) break;
        // publish this node's candidates; the last member of the group merges them
        if (t < 32) a.cand[((int64_t)level * kTsMaxCand + node) * 32 + t] = s_win[t];
        __threadfence();
        __syncthreads();
        const int parent = node / kTsFan;
        const int members = min(kTsFan, count - parent * kTsFan);
        if (t == 0) {
            unsigned* ctr = a.counters + level * kTsMaxCand + parent;
            const unsigned prev = atomicAdd(ctr, 1u);
            s_last = prev == (unsigned)(members - 1);
            if (s_last) *ctr = 0u;  // every member has arrived: ready for the next launch
        }
        __syncthreads();
        if (!s_last) return;
        __threadfence();
#pragma unroll
        for (int r = 0; r < kTsRpt; ++r) {
            const int sidx = r * kTsThreads + t, mem = sidx >> 5;
            rid[r] = mem < members
                         ? __ldcg(a.cand + ((int64_t)level * kTsMaxCand + parent * kTsFan + mem) * 32 + (sidx & 31))
                         : -1;
        }
#pragma unroll
        for (int r = 0; r < kTsRpt; ++r) load_leaf_row(a.A, a.ld, rid[r], a.lc0, a.w, v[r]);
        node = parent;
        count = (int)ceil_div(count, kTsFan);
        ++level;
    }

    // ---- root: pivots s_win[0..w); rows of L\U from the multipliers and the published pivot rows
    const int lc0 = a.lc0, w = a.w;
    batched_copy<kTsThreads, 32 * 32 / kTsThreads, float>(t, 32 * 32,
        [&](int e) {
            const int j = e >> 5, k = e & 31;
            const int l = s_loc[j];
            float x = 0.f;
            if (j < w && l >= 0 && k < w) {
                if (k < j) {
                    x = __ldcg(a.lmul + k * kTsRows + l);
                } else {
                    const float4 f = s_g.u[j][(k - j) >> 2];
                    const int e4 = (k - j) & 3;
                    x = e4 == 0 ? f.x : e4 == 1 ? f.y : e4 == 2 ? f.z : f.w;
                }
            }
            return x;
        },
        [&](int e, float x) { s_lu[e >> 5][e & 31] = x; });
    __syncthreads();
    if (t < 32) {
        const bool bad = t < w && (s_win[t] < 0 || !(fabsf(s_lu[t][t]) > 10.0f / FLT_MAX));
        const unsigned bb = __ballot_sync(0xffffffffu, bad);
        if (t == 0) {
            s_bad = bb ? lc0 + __ffs(bb) : 0;
            if (bb) a.status[kInfo] = s_bad;
        }
        s_flag[t] = 0;
        s_rdiag[t] = t < w ? rcp_nr(s_lu[t][t]) : 0.f;
    }
    for (int e = t; e < 32 * 32; e += kTsThreads) {  // transposed triangles for the substitutions
        const int i = e >> 5, k = e & 31;
        s_lt[i][k] = (k > i && k < w && i < w) ? s_lu[k][i] : 0.f;
        s_ut[i][k] = (k < i && i < w) ? s_lu[k][i] : 0.f;
    }
    __syncthreads();
    if (s_bad) return;
    // row moves: top slot lc0+j <- winner j; the displaced top rows fill the winners' old slots
    if (t < 32) {
        const int lane = t;
        const int p = lane < w ? s_win[lane] : -1;
        if (lane < w && p < lc0 + w) s_flag[p - lc0] = 1;
        __syncwarp();
        const bool disp = lane < w && !s_flag[lane];
        const bool outw = lane < w && p >= lc0 + w;
        const bool mtop = lane < w && p != lc0 + lane;
        const unsigned bd = __ballot_sync(0xffffffffu, disp), bo = __ballot_sync(0xffffffffu, outw),
                       bt = __ballot_sync(0xffffffffu, mtop);
        const unsigned below = (1u << lane) - 1u;
        if (outw) s_outpos[__popc(bo & below)] = p;
        __syncwarp();
        const int ntop = __popc(bt);
        if (mtop) {
            const int k = __popc(bt & below);
            s_mdst[k] = lc0 + lane;
            s_msrc[k] = p;
        }
        if (disp) {
            const int k = __popc(bd & below);
            s_mdst[ntop + k] = s_outpos[k];
            s_msrc[ntop + k] = lc0 + lane;
        }
        if (lane == 0) { s_nm = ntop + __popc(bd); s_nout = __popc(bd); }
    }
    __syncthreads();
    const int nm = s_nm, nout = s_nout;
    if (t == 0) { a.moves[0] = nm; a.moves[1] = nout; }
    if (t < nm) { a.moves[2 + t] = s_mdst[t]; a.moves[66 + t] = s_msrc[t]; }
    // thread t owns column c = t of the outer panel.  It writes the top rows' final content
    // (original rows left of the leaf, L11\U11 inside it, U12 = L11^-1 * original rows right of
    // it), the column of M = [U11^-1 | U11^-1 U12] that the apply kernel multiplies by, and the
    // original content of the rows that leave the top block.  All loads are issued before use.
    const int lo = lc0 - a.oc0, pw = a.pw, c = t;
    if (c < pw) {
        const bool in_leaf = c >= lo && c < lo + w;
        const float* col = a.A + a.oc0 + c;
        float x[32], y[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) x[j] = (j < w && !in_leaf) ? col[(int64_t)s_win[j] * a.ld] : 0.f;
#pragma unroll
        for (int k = 0; k < 32; ++k) y[k] = k < nout ? col[(int64_t)s_msrc[nm - nout + k] * a.ld] : 0.f;
#pragma unroll
        for (int k = 0; k < 32; ++k)
            if (k < nout) a.mvals[k * kNB + c] = y[k];
        if (in_leaf) {  // the top rows get L11\U11; x becomes e_(c-lo), for column c-lo of L11^-1
#pragma unroll
            for (int j = 0; j < 32; ++j)
                if (j < w) a.top[j * kNB + c] = s_lu[j][c - lo];
#pragma unroll
            for (int j = 0; j < 32; ++j) x[j] = j == c - lo ? 1.f : 0.f;
        }
        if (c >= lo) {
            // x <- L11^-1 x: column j of L read as float4s of its transposed copy
#pragma unroll
            for (int j = 0; j < 31; ++j) {
#pragma unroll
                for (int q = (j + 1) >> 2; q < 8; ++q) {
                    const float4 l4 = *reinterpret_cast<const float4*>(&s_lt[j][4 * q]);
                    const float lk[4] = {l4.x, l4.y, l4.z, l4.w};
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                        if (4 * q + e > j) x[4 * q + e] = fmaf(-lk[e], x[j], x[4 * q + e]);
                }
            }
        }
        if (in_leaf) {  // L11^-1 of the leaf, for the panel's triangular solve (lu_outer_kernel)
#pragma unroll
            for (int j = 0; j < 32; ++j) a.lpinv[((lo >> 5) * 32 + j) * 32 + (c - lo)] = j < w ? x[j] : 0.f;
        } else {
#pragma unroll
            for (int j = 0; j < 32; ++j)
                if (j < w) a.top[j * kNB + c] = x[j];
        }
        if (c >= lo) {
            // z = U11^-1 e_(c-lo) in the leaf, z = U11^-1 U12(:, c) right of it (back substitution)
            float z[32];
#pragma unroll
            for (int i = 0; i < 32; ++i) z[i] = in_leaf ? (i == c - lo ? 1.f : 0.f) : x[i];
#pragma unroll
            for (int i = 31; i >= 0; --i) {
                z[i] *= s_rdiag[i];
#pragma unroll
                for (int q = 0; q < (i + 3) / 4; ++q) {
                    const float4 u4 = *reinterpret_cast<const float4*>(&s_ut[i][4 * q]);
                    const float uk[4] = {u4.x, u4.y, u4.z, u4.w};
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                        if (4 * q + e < i) z[4 * q + e] = fmaf(-uk[e], z[i], z[4 * q + e]);
                }
            }
#pragma unroll
            for (int i = 0; i < 32; ++i)
                if (i < w) a.wmat[i * kNB + c] = z[i];
        }
    }
}

struct ApArgs {
    float* A;
    int64_t ld;
    int n, lc0, w, oc0, pw;
    const float* top;
    const float* mvals;
    const float* wmat;
    const int* moves;
    int32_t* perm;
    int32_t* pmap;  // the panel's row map: row i now holds what row pmap[i] held at the panel's start
    const int32_t* status;
    int nR;
};

// Applies a leaf: rows of the leaf's top block get their final content; every other row r below
// it (moved in from the side buffer or in place) becomes [v_left | l | v_right - l U12] with
// l = v_leaf U11^-1, computed as the product v_leaf * [U11^-1 | U11^-1 U12] (thread per column).
// The row moves are recorded in perm and in the panel's row map; the columns outside the outer
// panel are permuted once per panel (panel_permute_kernel).
__global__ void __launch_bounds__(256, 2) tslu_apply_kernel(ApArgs a) {
    __shared__ __align__(16) float s_l[kApRows][36];  // the rows' leaf values v_leaf
    __shared__ int s_mdst[64], s_msrc[64], s_src[kApRows];
    if (a.status[kInfo] != 0) return;
    const int t = threadIdx.x;
    const int nm = a.moves[0], nout = a.moves[1];
    if (t < nm) { s_mdst[t] = a.moves[2 + t]; s_msrc[t] = a.moves[66 + t]; }
    __syncthreads();
    if (blockIdx.x == 0 && a.perm) {
        int pv = 0, qv = 0;
        if (t < nm) { pv = a.perm[s_msrc[t]]; qv = a.pmap[s_msrc[t]]; }
        __syncthreads();
        if (t < nm) { a.perm[s_mdst[t]] = pv; a.pmap[s_mdst[t]] = qv; }
    }
    const int lo = a.lc0 - a.oc0, w = a.w, pw = a.pw, lc0 = a.lc0;
    const int r0 = lc0 + blockIdx.x * kApRows;
    const int nrows = min(kApRows, a.n - r0);
    if (t < kApRows) {
        const int i = r0 + t;
        int s = -1;                   // -1 own row, -2 top row, k >= 0 mvals[k]
        if (i < lc0 + w) {
            s = -2;
        } else {
            for (int k = 0; k < nout; ++k)
                if (s_mdst[nm - nout + k] == i) s = k;
        }
        s_src[t] = s;
    }
    __syncthreads();
    // thread t owns column c = t of the outer panel
    const int c = t;
    const bool active = c < pw;
    const bool in_leaf = c >= lo && c < lo + w;
    float x[kApRows], m[32];
#pragma unroll
    for (int r = 0; r < kApRows; ++r) {
        const int s = r < nrows ? s_src[r] : -1;
        const float* p = s == -2 ? a.top + (r0 + r - lc0) * kNB + c
                         : s >= 0 ? a.mvals + s * kNB + c
                                  : a.A + (int64_t)(r0 + r) * a.ld + a.oc0 + c;
        x[r] = (active && r < nrows && (s != -1 || c >= lo)) ? *p : 0.f;
    }
#pragma unroll
    for (int k = 0; k < 32; ++k) m[k] = (active && c >= lo && k < w) ? a.wmat[k * kNB + c] : 0.f;
    if (in_leaf) {
#pragma unroll
        for (int r = 0; r < kApRows; ++r) s_l[r][c - lo] = x[r];
    }
    if (t < kApRows * 4 && w < 32) {  // zero the unused leaf columns
        const int r = t >> 2;
        for (int k = w + (t & 3); k < 32; k += 4) s_l[r][k] = 0.f;
    }
    __syncthreads();
    if (!active) return;
    if (c >= lo) {
        const float sgn = in_leaf ? 1.f : -1.f;
#pragma unroll
        for (int r = 0; r < kApRows; ++r) {
            if (r >= nrows || s_src[r] == -2) continue;
            float acc = 0.f;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const float4 lv = *reinterpret_cast<const float4*>(&s_l[r][4 * q]);
                acc = fmaf(lv.x, m[4 * q], acc);
                acc = fmaf(lv.y, m[4 * q + 1], acc);
                acc = fmaf(lv.z, m[4 * q + 2], acc);
                acc = fmaf(lv.w, m[4 * q + 3], acc);
            }
            x[r] = in_leaf ? acc : fmaf(sgn, acc, x[r]);
        }
    }
#pragma unroll
    for (int r = 0; r < kApRows; ++r) {
        const int s = r < nrows ? s_src[r] : -1;
        if (r < nrows && (s != -1 || c >= lo)) a.A[(int64_t)(r0 + r) * a.ld + a.oc0 + c] = x[r];
    }
}

// U12 = L11^-1 A12 for the rows of the outer panel and the columns right of it (32-column strips),
// plus the K-major copies of U12 (and for 3xTF32 of L21) that the trailing GEMM reads.
struct OuArgs {
    float* A;
    int64_t ld;
    int n, oc0, pw, mode, nU;
    int cs0, ncols;  // trailing columns [oc0 + pw + cs0, + ncols) of U12 (the L21 split covers all rows)
    float* bth;
    float* btl;
    float* ah;
    float* al;
    const float* lpinv;  // [kNB / 32][32][32] inverses of the panel's diagonal 32 x 32 blocks of L
    const int32_t* status;
};

__device__ __forceinline__ float tf32_hi(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }

__global__ void __launch_bounds__(256) lu_outer_kernel(OuArgs a) {
    extern __shared__ float sm[];
    if (a.status[kInfo] != 0) return;
    const int t = threadIdx.x;
    const int c_first = a.oc0 + a.pw;  // first trailing column / row
    if (blockIdx.x >= a.nU) {
        // L21 split for 3xTF32: rows [c_first, n) x panel columns -> (ah, al) with row stride pw
        const int64_t e0 = ((int64_t)(blockIdx.x - a.nU) * 256 + t) * 4;
        const int64_t total = (int64_t)(a.n - c_first) * a.pw;
        if (e0 >= total) return;
        const int64_t r = e0 / a.pw;
        const int k = (int)(e0 - r * a.pw);
        const float4 x = *reinterpret_cast<const float4*>(a.A + (c_first + r) * a.ld + a.oc0 + k);
        const float4 h = make_float4(tf32_hi(x.x), tf32_hi(x.y), tf32_hi(x.z), tf32_hi(x.w));
        *reinterpret_cast<float4*>(a.ah + e0) = h;
        *reinterpret_cast<float4*>(a.al + e0) = make_float4(x.x - h.x, x.y - h.y, x.z - h.z, x.w - h.w);
        return;
    }
    const int pw = a.pw;
    const int cs = c_first + a.cs0 + blockIdx.x * 32;
    const int ncol = min(32, min(a.n, c_first + a.cs0 + a.ncols) - cs);
    float* s_x = sm;                  // [kNB][33] the strip (thread c owns column c)
    float* s_l = sm + kNB * 33;       // [kNB][36] one 32-column block of L (rows from the block down)
    float* s_li = s_l + kNB * 36;     // [32][36] the inverse of its diagonal block
    const int c = t & 31, rg = t >> 5;
    {
        float tmp[kNB / 8];
#pragma unroll
        for (int i = 0; i < kNB / 8; ++i) {
            const int r = rg + 8 * i;
            tmp[i] = (r < pw && c < ncol) ? a.A[(int64_t)(a.oc0 + r) * a.ld + cs + c] : 0.f;
        }
#pragma unroll
        for (int i = 0; i < kNB / 8; ++i) s_x[(rg + 8 * i) * 33 + c] = tmp[i];
    }
    // the next L block is loaded into registers while the current one is used
    float nl[kNB / 8], ni[4];
    auto load_block = [&](int b0) {
        const int bw = min(32, pw - b0);
#pragma unroll
        for (int i = 0; i < kNB / 8; ++i) {
            const int r = b0 + rg + 8 * i;
            nl[i] = (r < pw && c < bw) ? a.A[(int64_t)(a.oc0 + r) * a.ld + a.oc0 + b0 + c] : 0.f;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) ni[i] = a.lpinv[(b0 >> 5) * 1024 + (rg + 8 * i) * 32 + c];
    };
    load_block(0);
    for (int b0 = 0; b0 < pw; b0 += 32) {
        const int bw = min(32, pw - b0);
        __syncthreads();  // the previous block is no longer read
#pragma unroll
        for (int i = 0; i < kNB / 8; ++i)
            if (b0 + rg + 8 * i < pw) s_l[(rg + 8 * i) * 36 + c] = nl[i];
#pragma unroll
        for (int i = 0; i < 4; ++i) s_li[(rg + 8 * i) * 36 + c] = ni[i];
        __syncthreads();
        if (b0 + 32 < pw) load_block(b0 + 32);
        // x_b <- L_bb^-1 x_b: the block's 32 values of column c in registers, thread (c, rg) forms
        // rows rg + 8 q; the inverse's rows are read as float4 broadcasts
        float xb[32];
#pragma unroll
        for (int k = 0; k < 32; ++k) xb[k] = s_x[(b0 + k) * 33 + c];
        float y[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float4* li = reinterpret_cast<const float4*>(s_li + (rg + 8 * q) * 36);
            float acc = 0.f;
#pragma unroll
            for (int kq = 0; kq < 8; ++kq) {
                const float4 l4 = li[kq];
                acc = fmaf(l4.x, xb[4 * kq], acc);
                acc = fmaf(l4.y, xb[4 * kq + 1], acc);
                acc = fmaf(l4.z, xb[4 * kq + 2], acc);
                acc = fmaf(l4.w, xb[4 * kq + 3], acc);
            }
            y[q] = acc;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (rg + 8 * q < bw) s_x[(b0 + rg + 8 * q) * 33 + c] = y[q];
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 32; ++k) xb[k] = s_x[(b0 + k) * 33 + c];
        // rows below the block: x_r -= L(r, block) x_b, one float4 broadcast per 4 multipliers
        for (int r = b0 + bw + rg; r < pw; r += 8) {
            const float4* lr = reinterpret_cast<const float4*>(s_l + (r - b0) * 36);
            float acc = s_x[r * 33 + c];
#pragma unroll
            for (int kq = 0; kq < 8; ++kq) {
                const float4 l4 = lr[kq];
                acc = fmaf(-l4.x, xb[4 * kq], acc);
                acc = fmaf(-l4.y, xb[4 * kq + 1], acc);
                acc = fmaf(-l4.z, xb[4 * kq + 2], acc);
                acc = fmaf(-l4.w, xb[4 * kq + 3], acc);
            }
            s_x[r * 33 + c] = acc;
        }
    }
    __syncthreads();
    for (int r = rg; r < pw; r += 8)
        if (c < ncol) a.A[(int64_t)(a.oc0 + r) * a.ld + cs + c] = s_x[r * 33 + c];
    // Bt[col][k] = U12[k][col] (K-major), split for 3xTF32
    for (int cc = 0; cc < ncol; ++cc) {
        const int64_t o = (int64_t)(cs - c_first + cc) * pw;
        for (int k = t; k < pw; k += 256) {
            const float x = s_x[k * 33 + cc];
            if (a.mode == 3) {
                const float h = tf32_hi(x);
                a.bth[o + k] = h;
                a.btl[o + k] = x - h;
            } else {
                a.bth[o + k] = x;
            }
        }
    }
}

__global__ void iota_f32_kernel(int32_t* v, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = (int32_t)i;
}

// Inverses of the diagonal blocks (nb x nb) of the unit-lower L (which 0) and of U (which 1), used
// by the blocked triangular solves of the refinement.  One CTA per (block, triangle), thread per
// column of the inverse; the block and the growing inverse live in shared memory.
__global__ void diag_inv_kernel(const float* LU, int64_t ld, int n, int nb, float* linv, float* uinv,
                                const int32_t* status) {
    extern __shared__ float sm[];
    if (status[kInfo] != 0) return;
    const int blk = blockIdx.x >> 1, upper = blockIdx.x & 1;
    const int b0 = blk * nb, bs = min(nb, n - b0);
    const int SP = nb + 1;
    float* s_t = sm;             // [nb][SP] the triangle
    float* s_x = sm + nb * SP;   // [nb][SP] the inverse, column c owned by thread c
    const int c = threadIdx.x;
    if (c < bs)
        batched_copy<1, 16, float>(0, bs, [&](int r) { return LU[(int64_t)(b0 + r) * ld + b0 + c]; },
                                   [&](int r, float v) { s_t[r * SP + c] = v; });
    __syncthreads();
    if (c < nb) {
        if (!upper) {
            for (int i = 0; i < nb; ++i) {
                float acc = (i == c) ? 1.f : 0.f;
                if (i < bs)
                    for (int k = 0; k < i; ++k) acc = fmaf(-s_t[i * SP + k], s_x[k * SP + c], acc);
                s_x[i * SP + c] = (i < c || i >= bs) ? 0.f : acc;
            }
        } else {
            for (int i = nb - 1; i >= 0; --i) {
                float v = 0.f;
                if (i < bs && i <= c && c < bs) {
                    float acc = (i == c) ? 1.f : 0.f;
                    for (int k = i + 1; k <= c; ++k) acc = fmaf(-s_t[i * SP + k], s_x[k * SP + c], acc);
                    v = acc / s_t[i * SP + i];
                }
                s_x[i * SP + c] = v;
            }
        }
    }
    __syncthreads();
    float* out = (upper ? uinv : linv) + (int64_t)blk * nb * nb;
    for (int r = 0; r < nb; ++r)
        if (c < nb) out[r * nb + c] = s_x[r * SP + c];
}

// Coupling blocks of the persistent triangular sweeps: W_b = L_bb^-1 L_{b,b-1} (which 0, b >= 1) and
// W_b = U_bb^-1 U_{b,b+1} (which 1, b <= nblk - 2), 128 x 128 each, zero padded past the matrix.
// One CTA per (block, triangle); thread t owns rows 8 (t / 16) + [0, 8) and columns t % 16 + 16 [0, 8).
constexpr int kCpPitch = kTrsvNB + 1;
constexpr int kCpSmem = 2 * kTrsvNB * kCpPitch * (int)sizeof(float);
__global__ void __launch_bounds__(256) coupling_kernel(const float* LU, int64_t ld, int n, const float* linv,
                                                       const float* uinv, float* wl, float* wu, const int32_t* status) {
    extern __shared__ float sm[];
    if (status[kInfo] != 0) return;
    const int NB = kTrsvNB;
    const int nblk = (n + NB - 1) / NB;
    const int blk = blockIdx.x >> 1, upper = blockIdx.x & 1;
    if (upper ? blk >= nblk - 1 : blk == 0) return;
    const int b0 = blk * NB, bs = min(NB, n - b0);
    const int p0 = upper ? b0 + NB : b0 - NB, ps = min(NB, n - p0);
    float* s_i = sm;                 // [128][kCpPitch] T_bb^-1
    float* s_t = sm + NB * kCpPitch; // [128][kCpPitch] T_{b,p}
    const float* inv = (upper ? uinv : linv) + (int64_t)blk * NB * NB;
    const int t = threadIdx.x;
    batched_copy<256, 8, float>(t, NB * NB, [&](int e) { return inv[e]; },
                                [&](int e, float v) { s_i[(e >> 7) * kCpPitch + (e & (NB - 1))] = v; });
    batched_copy<256, 8, float>(t, NB * NB,
        [&](int e) {
            const int r = e >> 7, c = e & (NB - 1);
            return (r < bs && c < ps) ? LU[(int64_t)(b0 + r) * ld + p0 + c] : 0.f;
        },
        [&](int e, float v) { s_t[(e >> 7) * kCpPitch + (e & (NB - 1))] = v; });
    __syncthreads();
    const int r0 = 8 * (t >> 4), c0 = t & 15;
    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.f;
#pragma unroll 2
    for (int k = 0; k < NB; ++k) {
        float iv[8], tv[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) iv[i] = s_i[(r0 + i) * kCpPitch + k];
#pragma unroll
        for (int j = 0; j < 8; ++j) tv[j] = s_t[k * kCpPitch + c0 + 16 * j];
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(iv[i], tv[j], acc[i][j]);
    }
    float* out = (upper ? wu : wl) + (int64_t)blk * NB * NB;
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) out[(r0 + i) * NB + c0 + 16 * j] = acc[i][j];
}

// The outer panel's net row permutation applied to the columns [col_begin, col_end) (outside the
// panel): row i of the panel's rows [oc0, n) receives what row pmap[i] held when the panel started.
// CTA per 32 columns.  Each CTA lists the moved rows (at most 64 per leaf; warp-aggregated appends)
// and loads all of their sources into registers before any write.
constexpr int kPmMax = 64 * (kNB / 32);
__global__ void __launch_bounds__(256) panel_permute_kernel(float* A, int64_t ld, int n, int oc0, int col_begin,
                                                            int col_end, const int32_t* pmap, int32_t* status) {
    __shared__ int s_dst[kPmMax], s_src[kPmMax], s_cnt;
    if (status[kInfo] != 0) return;
    const int t = threadIdx.x, lane = t & 31;
    if (t == 0) s_cnt = 0;
    __syncthreads();
    constexpr int kScan = 16;  // row-map entries per thread per pass, all loaded before use
    for (int p0 = oc0; p0 < n; p0 += 256 * kScan) {
        int src[kScan];
#pragma unroll
        for (int u = 0; u < kScan; ++u) {
            const int i = p0 + 256 * u + t;
            src[u] = i < n ? pmap[i] : i;
        }
#pragma unroll
        for (int u = 0; u < kScan; ++u) {
            const int i = p0 + 256 * u + t;
            const bool mv = src[u] != i;
            const unsigned bal = __ballot_sync(0xffffffffu, mv);
            if (!bal) continue;  // warp-uniform
            int base = 0;
            if (lane == 0) base = atomicAdd(&s_cnt, __popc(bal));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (mv) {
                const int k = base + __popc(bal & ((1u << lane) - 1u));
                if (k < kPmMax) { s_dst[k] = i; s_src[k] = src[u]; }
            }
        }
    }
    __syncthreads();
    const int cnt = s_cnt;
    if (cnt > kPmMax) {  // cannot happen: each leaf moves at most 64 rows
        if (t == 0) atomicExch(&status[kTimeout], 401);
        return;
    }
    const int col = col_begin + blockIdx.x * 32 + (t & 31), rg = t >> 5;
    const bool ok = col < col_end && col < n;
    float x[kPmMax / 8];
#pragma unroll
    for (int q = 0; q < kPmMax / 8; ++q) {
        const int k = rg + 8 * q;
        x[q] = (ok && k < cnt) ? A[(int64_t)s_src[k] * ld + col] : 0.f;
    }
    __syncthreads();  // every source of this CTA's columns is read before any row is written
#pragma unroll
    for (int q = 0; q < kPmMax / 8; ++q) {
        const int k = rg + 8 * q;
        if (ok && k < cnt) A[(int64_t)s_dst[k] * ld + col] = x[q];
    }
}

}  // namespace

// Scratch of the FP32 factorisation (all device memory, carved from one workspace).
size_t f32_scratch_bytes(int64_t n) {
    const int64_t nblk = ceil_div(n, kTrsvNB);
    size_t b = 0;
    b += (size_t)kTsLevels * kTsMaxCand * 32 * sizeof(int);   // cand
    b += (size_t)kTsLevels * kTsMaxCand * sizeof(unsigned);   // counters
    b += 3 * 32 * kNB * sizeof(float);                          // top, mvals, wmat
    b += 256 * sizeof(int);                                     // moves
    b += 32 * (size_t)kTsRows * sizeof(float);                  // root multipliers
    b += 2 * (size_t)round_up(n, 64) * sizeof(int32_t);          // panel row maps (by panel parity)
    b += 2 * (size_t)kNB * 32 * sizeof(float);                  // leaf L11^-1 blocks (by panel parity)
    b += 4 * (size_t)round_up(n, 32) * kNB * sizeof(float);     // bth, btl, ah, al
    b += 4 * (size_t)nblk * kTrsvNB * kTrsvNB * sizeof(float);  // diagonal inverses, coupling blocks
    b += 2 * (size_t)nblk * kSweepGroups * kTrsvNB * 8 * sizeof(unsigned long long);  // sweep words
    return b + 16 * 256;
}

F32Scratch f32_scratch_carve(void* base, int64_t n) {
    F32Scratch s;
    char* p = static_cast<char*>(base);
    auto take = [&](size_t bytes) {
        char* q = p;
        p += round_up((int64_t)bytes, 256);
        return q;
    };
    const int64_t nblk = ceil_div(n, kTrsvNB);
    s.cand = reinterpret_cast<int*>(take((size_t)kTsLevels * kTsMaxCand * 32 * sizeof(int)));
    s.counters = reinterpret_cast<unsigned*>(take((size_t)kTsLevels * kTsMaxCand * sizeof(unsigned)));
    s.counters_bytes = (size_t)kTsLevels * kTsMaxCand * sizeof(unsigned);
    s.top = reinterpret_cast<float*>(take(32 * kNB * sizeof(float)));
    s.mvals = reinterpret_cast<float*>(take(32 * kNB * sizeof(float)));
    s.wmat = reinterpret_cast<float*>(take(32 * kNB * sizeof(float)));
    s.moves = reinterpret_cast<int*>(take(256 * sizeof(int)));
    s.lmul = reinterpret_cast<float*>(take(32 * (size_t)kTsRows * sizeof(float)));
    s.pmap = reinterpret_cast<int32_t*>(take(2 * (size_t)round_up(n, 64) * sizeof(int32_t)));
    s.lpinv = reinterpret_cast<float*>(take(2 * (size_t)kNB * 32 * sizeof(float)));
    const size_t panel = (size_t)round_up(n, 32) * kNB * sizeof(float);
    s.bth = reinterpret_cast<float*>(take(panel));
    s.btl = reinterpret_cast<float*>(take(panel));
    s.ah = reinterpret_cast<float*>(take(panel));
    s.al = reinterpret_cast<float*>(take(panel));
    s.linv = reinterpret_cast<float*>(take((size_t)nblk * kTrsvNB * kTrsvNB * sizeof(float)));
    s.uinv = reinterpret_cast<float*>(take((size_t)nblk * kTrsvNB * kTrsvNB * sizeof(float)));
    s.wl = reinterpret_cast<float*>(take((size_t)nblk * kTrsvNB * kTrsvNB * sizeof(float)));
    s.wu = reinterpret_cast<float*>(take((size_t)nblk * kTrsvNB * kTrsvNB * sizeof(float)));
    s.ll = reinterpret_cast<unsigned long long*>(
        take(2 * (size_t)nblk * kSweepGroups * kTrsvNB * 8 * sizeof(unsigned long long)));
    return s;
}

int32_t lu_factor_f32(Ctx* ctx, cudaStream_t st, float* A, int64_t ld, int64_t n, int32_t* perm, int mode,
                      const F32Scratch& s) {
    if (n <= 0) return B2M_OK;
    if ((ld & 31) || (reinterpret_cast<uintptr_t>(A) & 127))
        return fail(ctx, B2M_ERR_DIM, "lu_factor_f32: ld must be a multiple of 32 floats, A 128-byte aligned");
    if (n > (int64_t)kTsMaxCand * kTsRows) return fail(ctx, B2M_ERR_UNSUPPORTED, "mixed LU: n too large");
    std::atomic<int>& attr = device_flag((const void*)lu_outer_kernel, 0, ctx->device);
    const int ou_smem = (kNB * 33 + (kNB + 32) * 36) * sizeof(float);
    const int di_smem = 2 * kTrsvNB * (kTrsvNB + 1) * sizeof(float);
    if (!attr.load()) {
        B2M_CU(ctx, cudaFuncSetAttribute(lu_outer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, ou_smem));
        B2M_CU(ctx, cudaFuncSetAttribute(diag_inv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, di_smem));
        B2M_CU(ctx, cudaFuncSetAttribute(coupling_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kCpSmem));
        // one shared-memory carveout for every kernel of the factorisation, so that the panel kernels
        // can share SMs with the tiles of a concurrent trailing GEMM (which needs the maximum)
        for (const void* f : {(const void*)tslu_select_kernel, (const void*)tslu_apply_kernel,
                              (const void*)panel_permute_kernel, (const void*)lu_outer_kernel})
            B2M_CU(ctx, cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout,
                                             (int)cudaSharedmemCarveoutMaxShared));
        attr.store(1);
    }
    B2M_TRY(ensure_side_stream(ctx));
    const GraphKey key0{3 + mode * 10, A, perm, s.cand, s.bth, ld, n, 0, 1};
    const GraphKey key1{3 + mode * 10, A, perm, s.cand, s.bth, ld, n, 0, 2};
    // part 0: the first outer panel's leaves; part 1: everything after them.  Two graphs, so that the
    // device factors the first panel while the host still submits the large second graph (a graph's
    // launch costs host time per node).
    auto issue = [&](cudaStream_t q, int part) -> int32_t {
        // Look-ahead: after a panel, only the next panel's columns are updated on this stream; the
        // rest of the trailing update runs on the side stream, overlapping the next panel's leaves
        // (which touch neither those columns nor the previous panel's L21), and is joined before
        // the next panel's out-of-panel row permutation.  The leaf kernels carry the highest
        // priority so that they take SMs ahead of the wide GEMM's tiles.
        cudaStream_t q2 = ctx->side_stream;
        bool side_busy = false;
        PriorityScope hi(ctx, true);  // launch_k launches on this stream are the critical path
        cudaLaunchAttribute pri[1];
        pri[0].id = cudaLaunchAttributePriority;
        pri[0].val.priority = ctx->chain_priority;
        auto cfg_of = [&](unsigned grid, unsigned block, size_t smem) {
            cudaLaunchConfig_t c{};
            c.gridDim = dim3(grid);
            c.blockDim = dim3(block);
            c.dynamicSmemBytes = smem;
            c.stream = q;
            c.attrs = pri;
            c.numAttrs = ctx->launch_hi ? 1 : 0;  // the side stream's launches (PriorityScope) go without
            return c;
        };
        if (part == 0) {
            B2M_CU(ctx, cudaMemsetAsync(s.counters, 0, s.counters_bytes, q));
            iota_f32_kernel<<<(unsigned)ceil_div(n, 256), 256, 0, q>>>(perm, n);
            B2M_LAUNCHED(ctx);
        }
        for (int64_t oc0 = 0; oc0 < n; oc0 += kNB) {
            const int pw = (int)std::min<int64_t>(kNB, n - oc0);
            // the row map alternates between two buffers by panel parity: the side stream may still
            // be permuting the previous panel's left columns with its map while this panel's first
            // leaf initialises the other one (the join below orders the reuse two panels later)
            int32_t* pmap = s.pmap + ((oc0 / kNB) & 1) * round_up(n, 64);
            // the leaves' L11^-1 blocks alternate the same way: the side stream's U12 of the columns
            // beyond the next panel still reads this panel's blocks while the next panel's leaves
            // write theirs (without the second buffer those reads raced with the writes)
            float* lpinv = s.lpinv + ((oc0 / kNB) & 1) * (size_t)kNB * 32;
            const bool leaves = (part == 0) == (oc0 == 0);
            for (int64_t lc0 = oc0; leaves && lc0 < oc0 + pw; lc0 += 32) {
                const int w = (int)std::min<int64_t>(32, n - lc0);
                TsArgs ta{A, ld, (int)n, (int)lc0, w, (int)oc0, pw, s.cand, s.counters, s.top, s.mvals, s.wmat,
                          s.moves, s.lmul, lc0 == oc0 ? pmap : nullptr, lpinv, ctx->d_status};
                prof_begin(ctx, q, kClsPanel);
                {
                    const cudaLaunchConfig_t c = cfg_of((unsigned)ceil_div(n - lc0, kTsRows), kTsThreads, 0);
                    B2M_CU(ctx, cudaLaunchKernelEx(&c, tslu_select_kernel, ta));
                }
                prof_end(ctx, q, kClsPanel, 4.0 * (n - lc0) * 32);  // bytes: the leaf's columns, read once
                B2M_LAUNCHED(ctx);
                ApArgs aa{A, ld, (int)n, (int)lc0, w, (int)oc0, pw, s.top, s.mvals, s.wmat, s.moves, perm, pmap,
                          ctx->d_status, 0};
                aa.nR = (int)ceil_div(n - lc0, kApRows);
                prof_begin(ctx, q, kClsSwap);
                {
                    const cudaLaunchConfig_t c = cfg_of((unsigned)aa.nR, 256, 0);
                    B2M_CU(ctx, cudaLaunchKernelEx(&c, tslu_apply_kernel, aa));
                }
                // bytes: the panel rows read and written
                prof_end(ctx, q, kClsSwap, 8.0 * (n - lc0) * (pw - (lc0 - oc0)));
                B2M_LAUNCHED(ctx);
            }
            if (part == 0) return B2M_OK;
            if (side_busy) {  // the previous panel's wide update must be done before rows move under it
                B2M_CU(ctx, cudaEventRecord(ctx->ev_side_join, q2));
                B2M_CU(ctx, cudaStreamWaitEvent(q, ctx->ev_side_join, 0));
                side_busy = false;
            }
            const int64_t c1 = oc0 + pw;
            auto permute = [&](cudaStream_t qs, int64_t c_begin, int64_t c_end) -> int32_t {
                if (c_end <= c_begin) return B2M_OK;
                cudaLaunchConfig_t c = cfg_of((unsigned)ceil_div(c_end - c_begin, 32), 256, 0);
                c.stream = qs;
                prof_begin(ctx, qs, kClsSwap);
                B2M_CU(ctx, cudaLaunchKernelEx(&c, panel_permute_kernel, A, ld, (int)n, (int)oc0, (int)c_begin,
                                               (int)c_end, (const int32_t*)pmap, ctx->d_status));
                // bytes: at most 64 moved rows per leaf, read and written
                prof_end(ctx, qs, kClsSwap, 8.0 * 64 * (pw / 32) * (double)(c_end - c_begin));
                B2M_LAUNCHED(ctx);
                return B2M_OK;
            };
            // Only the next panel's columns are on this stream's critical path: their permutation,
            // U12 block, the L21 split and their GEMM.  The other columns right of the panel (their
            // permutation, U12 and GEMM) and the factored columns on the left (their permutation)
            // go to the side stream, which is joined before the next panel's permutation.
            const int64_t M = n - c1;
            const int64_t nw = std::min<int64_t>(kNB, std::max<int64_t>(M, 0));  // the next panel's columns
            B2M_TRY(permute(q, c1, c1 + nw));
            if (c1 >= n) {
                if (oc0 > 0) {
                    B2M_CU(ctx, cudaEventRecord(ctx->ev_side_fork, q));
                    B2M_CU(ctx, cudaStreamWaitEvent(q2, ctx->ev_side_fork, 0));
                    PriorityScope side(ctx, false);
                    B2M_TRY(permute(q2, 0, oc0));
                    side_busy = true;
                }
                break;
            }
            const int nL = mode == 3 ? (int)ceil_div(M * pw, 1024) : 0;
            auto outer = [&](cudaStream_t qs, int64_t cs0, int64_t ncols, int nl) -> int32_t {
                OuArgs oa{A, ld, (int)n, (int)oc0, pw, mode, (int)ceil_div(ncols, 32), (int)cs0, (int)ncols,
                          s.bth, s.btl, s.ah, s.al, lpinv, ctx->d_status};
                prof_begin(ctx, qs, kClsTrsm);
                B2M_CU(ctx, launch_k(ctx, lu_outer_kernel, dim3((unsigned)(oa.nU + nl)), dim3(256), (size_t)ou_smem, qs, oa));
                // bytes: U12 read and written, its GEMM copies written, L21 read and split (3xTF32)
                prof_end(ctx, qs, kClsTrsm,
                         8.0 * pw * ncols + 4.0 * ncols * pw * (mode == 3 ? 2 : 1) + (nl ? 12.0 * M * pw : 0.0));
                B2M_LAUNCHED(ctx);
                return B2M_OK;
            };
            auto gemm = [&](cudaStream_t qs, int64_t cs0, int64_t ncols) -> int32_t {
                FOperand bh{s.bth, pw, M, pw, cs0, 0};
                float* C = A + c1 * ld + c1 + cs0;
                if (mode == 3) {
                    FOperand ah{s.ah, pw, M, pw, 0, 0};
                    return sgemm_tc(ctx, qs, ah, s.al, bh, s.btl, C, ld, M, ncols, pw, B2M_DO_SUB, 3, true);
                }
                FOperand ah{A, ld, n, n, c1, oc0};
                return sgemm_tc(ctx, qs, ah, nullptr, bh, nullptr, C, ld, M, ncols, pw, B2M_DO_SUB, 1, true);
            };
            B2M_TRY(outer(q, 0, nw, nL));  // with the L21 split that both GEMMs read
            if (M > nw || oc0 > 0) {
                B2M_CU(ctx, cudaEventRecord(ctx->ev_side_fork, q));
                B2M_CU(ctx, cudaStreamWaitEvent(q2, ctx->ev_side_fork, 0));
                PriorityScope side(ctx, false);
                if (M > nw) B2M_TRY(permute(q2, c1 + nw, n));
                if (oc0 > 0) B2M_TRY(permute(q2, 0, oc0));
                if (M > nw) {
                    B2M_TRY(outer(q2, nw, M - nw, 0));
                    B2M_TRY(gemm(q2, nw, M - nw));
                }
                side_busy = true;
            }
            B2M_TRY(gemm(q, 0, nw));
        }
        if (side_busy) {
            B2M_CU(ctx, cudaEventRecord(ctx->ev_side_join, q2));
            B2M_CU(ctx, cudaStreamWaitEvent(q, ctx->ev_side_join, 0));
        }
        const int nblk = (int)ceil_div(n, kTrsvNB);
        diag_inv_kernel<<<2 * nblk, kTrsvNB, di_smem, q>>>(A, ld, (int)n, kTrsvNB, s.linv, s.uinv, ctx->d_status);
        B2M_LAUNCHED(ctx);
        coupling_kernel<<<2 * nblk, 256, kCpSmem, q>>>(A, ld, (int)n, s.linv, s.uinv, s.wl, s.wu, ctx->d_status);
        B2M_LAUNCHED(ctx);
        return B2M_OK;
    };
    B2M_TRY(run_graph(ctx, st, key0, [&](cudaStream_t q) { return issue(q, 0); }));
    return run_graph(ctx, st, key1, [&](cudaStream_t q) { return issue(q, 1); });
}

}  // namespace b2m
