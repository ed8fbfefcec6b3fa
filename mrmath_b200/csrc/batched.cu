// batched.cu -- many independent LU solves of uneven order in one persistent launch.
//
// There is no counterpart in the reference, which solves one system per MatrixLinEQSolve call
// (LinAlgLU.pas:481-592); every system here follows that routine's semantics: partial pivoting with
// the first maximum winning, the pivot column scaled by the reciprocal of the pivot, a pivot of
// magnitude <= 10/MaxDouble reporting the system singular (:246-268), forward substitution with the
// unit-lower factor and back substitution dividing by U's diagonal (:315-385).
//
// Scheduling: the host sorts the systems largest first; resident CTAs pull them from an atomic work
// queue (longest-processing-time first, no tail of big systems).  Systems of order > small_n take
// a whole CTA; smaller ones are handed out in batches, one per group of G warps, each group with its
// own named barrier.  The panel width of both size buckets and G are chosen by the autotuner at the
// bottom of this file, which times the candidate shapes on the caller's batch.
//
// Per system: A is copied into the CTA's private scratch slice (<= 256 x 256, L2 resident), where
// a blocked right-looking LU runs with the current panel and the block row of U in shared memory.
// Rows are never moved: a permutation maps factor rows to storage rows, so a pivot interchange swaps
// two integers (the factors and the reference's interchange order are the same as with physical
// swaps).  The solve is blocked by 32 rows: one warp per right-hand side substitutes a diagonal
// block with shuffles, then the group folds it into the remaining rows.
//
// Mode 1 factors in FP32 and refines in FP64: r = b - A x from the caller's FP64 A, d from the FP32
// factors, x += d, until the normwise backward error max_q ||r_q|| / (||A|| ||x_q|| + ||b_q||) is
// <= n 2^-53; a stall or an FP32 pivot <= 10/FLT_MAX refactors that system in FP64.
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <climits>
#include <cstring>
#include <numeric>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace b2m {
namespace {

constexpr int kBThreads = 256;
constexpr int kBMaxN = 256;
constexpr int kBMaxK = 8;
constexpr int kBMaxPW = 32;
constexpr int kStrip = 2;  // 16 x 8 tiles per warp step of the trailing update

struct BatchArgs {
    int count;
    const int32_t* n;
    const int32_t* k;
    const int64_t* a_off;
    const int64_t* b_off;
    const double* A;
    const double* B;
    double* X;
    double* scratch;  // kBMaxN^2 doubles per CTA
    const int32_t* order;
    int32_t* counter;
    int32_t* info;
    int32_t* iters;
    int mode;
    int small_n;
    int group_warps;
    int big_warps;
    int pw_large, pw_small;
    int max_iter;
};

// a group of threads working on one system, with its own named barrier
struct Grp {
    int tid, nt, bar;
    __device__ __forceinline__ void sync() const { asm volatile("bar.sync %0, %1;\n" ::"r"(bar), "r"(nt) : "memory"); }
};

// shared-memory slice of one group
struct Slice {
    double* pan;   // [nmax][pw + 1] panel (factor rows c0.., panel columns)
    double* u;     // [pw][nmax + 1] block row of U right of the panel
    double* y;     // [nmax][kBMaxK] right-hand sides / solution in factor order
    double* red;   // [8] reduction values
    int* redi;     // [8] reduction indices
    int* perm;     // [nmax] storage row of factor row i
    int* flag;     // [4]
    int us;        // row stride of u
    int pw;        // panel width
};

__host__ __device__ inline size_t slice_doubles(int nmax, int pw) {
    return (size_t)nmax * (pw + 1) + (size_t)pw * (nmax + 1) + (size_t)nmax * kBMaxK + 8 + (nmax + 8 + 4 + 1) / 2 + 1;
}

__device__ Slice carve(double* base, int nmax, int pw) {
    Slice s;
    s.pan = base;
    s.u = s.pan + (size_t)nmax * (pw + 1);
    s.y = s.u + (size_t)pw * (nmax + 1);
    s.red = s.y + (size_t)nmax * kBMaxK;
    s.redi = reinterpret_cast<int*>(s.red + 8);
    s.perm = s.redi + 8;
    s.flag = s.perm + nmax;
    s.us = nmax + 1;
    s.pw = pw;
    return s;
}

// factor scratch of one CTA: a matrix of the slice's order per group
__host__ __device__ inline size_t batch_scratch_doubles(int small_n, int G, int GB) {
    const size_t big = (size_t)((kBThreads / 32) / GB) * kBMaxN * kBMaxN;
    const size_t small = (size_t)((kBThreads / 32) / G) * small_n * small_n;
    return big > small ? big : small;
}

template <typename T> __device__ __forceinline__ T sing_thresh();
template <> __device__ __forceinline__ double sing_thresh<double>() { return 10.0 / DBL_MAX; }
template <> __device__ __forceinline__ float sing_thresh<float>() { return 10.0f / FLT_MAX; }

// argmax of |v| over the group (first maximum wins: lowest index among equals); all threads get it
__device__ __forceinline__ void grp_argmax(const Grp& g, const Slice& s, double v, int i, double& bv, int& bi) {
    const int lane = g.tid & 31, w = g.tid >> 5, nw = g.nt >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double v2 = __shfl_xor_sync(0xffffffffu, v, o);
        const int i2 = __shfl_xor_sync(0xffffffffu, i, o);
        if (i2 >= 0 && (i < 0 || v2 > v || (v2 == v && i2 < i))) { v = v2; i = i2; }
    }
    if (nw == 1) {
        bv = v;
        bi = i;
        return;
    }
    if (lane == 0) { s.red[w] = v; s.redi[w] = i; }
    g.sync();
    bv = -1.0;
    bi = -1;
    for (int q = 0; q < nw; ++q) {
        const double v2 = s.red[q];
        const int i2 = s.redi[q];
        if (i2 >= 0 && (bi < 0 || v2 > bv || (v2 == bv && i2 < bi))) { bv = v2; bi = i2; }
    }
    g.sync();
}

// pivot search over the group: the largest candidate magnitude v >= 0, the lowest row index among
// equal magnitudes (the first maximum of the reference's scan).  A thread without a candidate
// passes v = 0 and i = INT_MAX.  Non-negative doubles order like their bit patterns, so the
// comparison runs on the 64-bit key as two 32-bit warp reductions, then a minimum over the
// indices of the lanes that hold the maximum; the warps' winners are combined the same way.
__device__ __forceinline__ void warp_pivot(double v, int i, double& bv, int& bi) {
    const unsigned long long key = (unsigned long long)__double_as_longlong(v);
    const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
    const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
    const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
    const unsigned mi = __reduce_min_sync(0xffffffffu, (hi == mhi && lo == mlo) ? (unsigned)i : 0xffffffffu);
    bv = __longlong_as_double((long long)(((unsigned long long)mhi << 32) | mlo));
    bi = (int)mi;
}

__device__ __forceinline__ void grp_pivot(const Grp& g, const Slice& s, double v, int i, double& bv, int& bi) {
    const int lane = g.tid & 31, w = g.tid >> 5, nw = g.nt >> 5;
    warp_pivot(v, i, bv, bi);
    if (nw == 1) return;
    if (lane == 0) { s.red[w] = bv; s.redi[w] = bi; }
    g.sync();
    warp_pivot(lane < nw ? s.red[lane] : 0.0, lane < nw ? s.redi[lane] : INT_MAX, bv, bi);
    g.sync();
}

// Blocked LU of the n x n matrix A0 (FP64, row-major, ld n) into W (element type T, same layout)
// with row permutation perm.  The first panel reads A0 directly and its updates write every entry
// of W, so A0 is never copied separately.  Global loads are issued in groups before they are used
// (a loop that loads, computes and stores one element at a time pays one L2 latency per element).
// Returns 0, or 1 when a pivot is <= the singular threshold (uniform across the group).
template <typename T>
__device__ int grp_lu(const Grp& g, const Slice& s, const double* A0, T* W, int n, int PW) {
    for (int i = g.tid; i < n; i += g.nt) s.perm[i] = i;
    g.sync();
    const int pwp = PW + 1;
    for (int c0 = 0; c0 < n; c0 += PW) {
        const bool first = c0 == 0;
        auto at = [&](int row, int col) -> T {
            return first ? (T)A0[(int64_t)row * n + col] : W[(int64_t)row * n + col];
        };
        const int pw = min(PW, n - c0), m = n - c0;
        // panel: one factor row per thread, all of its loads in flight
        for (int r = g.tid; r < m; r += g.nt) {
            const int row = s.perm[c0 + r];
            for (int cb = 0; cb < pw; cb += 8) {
                T v[8];
#pragma unroll
                for (int c = 0; c < 8; ++c)
                    if (cb + c < pw) v[c] = at(row, c0 + cb + c);
#pragma unroll
                for (int c = 0; c < 8; ++c)
                    if (cb + c < pw) s.pan[r * pwp + cb + c] = (double)v[c];
            }
        }
        g.sync();
        for (int j = 0; j < pw; ++j) {
            double v = -1.0;
            int vi = INT_MAX;
            for (int r = j + g.tid; r < m; r += g.nt) {
                const double a = fabs(s.pan[r * pwp + j]);
                if (a > v) { v = a; vi = r; }  // a NaN never wins
            }
            if (vi == INT_MAX) v = 0.0;
            double bv;
            int pr;
            grp_pivot(g, s, v, vi, bv, pr);
            if (!(bv > (double)sing_thresh<T>())) return 1;
            if (pr != j) {
                for (int c = g.tid; c < pw; c += g.nt) {
                    const double t0 = s.pan[j * pwp + c];
                    s.pan[j * pwp + c] = s.pan[pr * pwp + c];
                    s.pan[pr * pwp + c] = t0;
                }
                if (g.tid == 0) {
                    const int t1 = s.perm[c0 + j];
                    s.perm[c0 + j] = s.perm[c0 + pr];
                    s.perm[c0 + pr] = t1;
                }
            }
            g.sync();
            // reference scaling: the column is multiplied by 1/pivot, in the element type
            const T rinv = (T)1 / (T)s.pan[j * pwp + j];
            for (int r = j + 1 + g.tid; r < m; r += g.nt) {
                const T l = (T)s.pan[r * pwp + j] * rinv;
                s.pan[r * pwp + j] = (double)l;
                for (int c = j + 1; c < pw; ++c)
                    s.pan[r * pwp + c] = (double)((T)s.pan[r * pwp + c] - l * (T)s.pan[j * pwp + c]);
            }
            g.sync();
        }
        for (int r = g.tid; r < m; r += g.nt) {
            T* dst = W + (int64_t)s.perm[c0 + r] * n + c0;
            for (int c = 0; c < pw; ++c) dst[c] = (T)s.pan[r * pwp + c];
        }
        const int c1 = c0 + pw, nr = n - c1;
        if (nr > 0) {
            // block row of U: u = L11^-1 A12 (thread per column, loads in groups of 8)
            for (int c = g.tid; c < nr; c += g.nt) {
                for (int r0 = 0; r0 < pw; r0 += 8) {
                    T v[8];
#pragma unroll
                    for (int e = 0; e < 8; ++e)
                        if (r0 + e < pw) v[e] = at(s.perm[c0 + r0 + e], c1 + c);
#pragma unroll
                    for (int e = 0; e < 8; ++e)
                        if (r0 + e < pw) s.u[(r0 + e) * s.us + c] = (double)v[e];
                }
                W[(int64_t)s.perm[c0] * n + c1 + c] = (T)s.u[c];
                for (int r = 1; r < pw; ++r) {
                    T acc = (T)s.u[r * s.us + c];
                    for (int q = 0; q < r; ++q) acc -= (T)s.pan[r * pwp + q] * (T)s.u[q * s.us + c];
                    s.u[r * s.us + c] = (double)acc;
                    W[(int64_t)s.perm[c0 + r] * n + c1 + c] = acc;
                }
            }
            g.sync();
            if constexpr (std::is_same<T, double>::value) {
                // trailing update A22 -= L21 U12 on the FP64 tensor cores: warps walk 16 x 8 tiles;
                // m16n8k4 fragments (g = lane / 4, t = lane % 4): a = (L21[g][k+t], L21[g+8][k+t]),
                // b = U12[k+t][g], c = C[g][2t..2t+1], C[g+8][2t..2t+1]
                // A warp takes a 16 x 8 kStrip strip (kStrip 16 x 8 tiles sharing the L21
                // fragment), so that its 4 kStrip loads of C are in flight together.
                const int lane = g.tid & 31, nw = g.nt >> 5, gq = lane >> 2, tq = lane & 3;
                const int tm = (nr + 15) / 16, tn = (nr + 8 * kStrip - 1) / (8 * kStrip);
                for (int tile = g.tid >> 5; tile < tm * tn; tile += nw) {
                    const int r0 = (tile / tn) * 16, q0 = (tile % tn) * 8 * kStrip;
                    const int ra = r0 + gq, rb = r0 + gq + 8;
                    const bool oka = ra < nr, okb = rb < nr;
                    const int rowa = oka ? s.perm[c1 + ra] : 0, rowb = okb ? s.perm[c1 + rb] : 0;
                    double d[kStrip][4];
#pragma unroll
                    for (int u = 0; u < kStrip; ++u) {
                        const int cc = q0 + 8 * u + 2 * tq;
                        d[u][0] = (oka && cc < nr) ? (double)at(rowa, c1 + cc) : 0.0;
                        d[u][1] = (oka && cc + 1 < nr) ? (double)at(rowa, c1 + cc + 1) : 0.0;
                        d[u][2] = (okb && cc < nr) ? (double)at(rowb, c1 + cc) : 0.0;
                        d[u][3] = (okb && cc + 1 < nr) ? (double)at(rowb, c1 + cc + 1) : 0.0;
                    }
                    const double* la = s.pan + (pw + min(ra, nr - 1)) * pwp;
                    const double* lb = s.pan + (pw + min(rb, nr - 1)) * pwp;
                    for (int k = 0; k < pw; k += 4) {
                        const int kk = k + tq;
                        const double a0 = kk < pw ? -la[kk] : 0.0;
                        const double a1 = kk < pw ? -lb[kk] : 0.0;
#pragma unroll
                        for (int u = 0; u < kStrip; ++u) {
                            const int cb = min(q0 + 8 * u + gq, nr - 1);
                            const double b0 = kk < pw ? s.u[kk * s.us + cb] : 0.0;
                            asm volatile(
                                "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
                                "{%0,%1,%2,%3};\n"
                                : "+d"(d[u][0]), "+d"(d[u][1]), "+d"(d[u][2]), "+d"(d[u][3])
                                : "d"(a0), "d"(a1), "d"(b0));
                        }
                    }
                    const int64_t oa = (int64_t)rowa * n + c1, ob = (int64_t)rowb * n + c1;
#pragma unroll
                    for (int u = 0; u < kStrip; ++u) {
                        const int cc = q0 + 8 * u + 2 * tq;
                        if (oka && cc < nr) W[oa + cc] = (T)d[u][0];
                        if (oka && cc + 1 < nr) W[oa + cc + 1] = (T)d[u][1];
                        if (okb && cc < nr) W[ob + cc] = (T)d[u][2];
                        if (okb && cc + 1 < nr) W[ob + cc + 1] = (T)d[u][3];
                    }
                }
            } else {
            // trailing update A22 -= L21 U12: thread per column, 8 rows per step, loads first
            for (int c = g.tid; c < nr; c += g.nt) {
                for (int r0 = 0; r0 < nr; r0 += 8) {
                    T v[8];
#pragma unroll
                    for (int e = 0; e < 8; ++e) v[e] = r0 + e < nr ? at(s.perm[c1 + r0 + e], c1 + c) : (T)0;
                    for (int q = 0; q < pw; ++q) {
                        const T uq = (T)s.u[q * s.us + c];
#pragma unroll
                        for (int e = 0; e < 8; ++e) v[e] -= (T)s.pan[min(pw + r0 + e, m - 1) * pwp + q] * uq;
                    }
#pragma unroll
                    for (int e = 0; e < 8; ++e)
                        if (r0 + e < nr) W[(int64_t)s.perm[c1 + r0 + e] * n + c1 + c] = v[e];
                }
            }
            }
            g.sync();
        }
    }
    return 0;
}

// y (factor order, kk columns) <- U^-1 L^-1 y with the factors in W (element type T).  Each
// 32-row diagonal block is staged in shared memory (over the then idle panel / U buffers); one warp
// per right-hand side substitutes it with shuffles, then the group folds it into the other rows.
template <typename T>
__device__ void grp_solve(const Grp& g, const Slice& s, const T* W, int n, int kk) {
    const int lane = g.tid & 31, w = g.tid >> 5, nw = g.nt >> 5;
    const int nb = (n + 31) / 32;
    double* blk = s.pan;  // [32][33], spans into the U buffer for narrow panels
    for (int pass = 0; pass < 2; ++pass) {
        const bool lower = pass == 0;
        for (int bi = 0; bi < nb; ++bi) {
            const int b = lower ? bi : nb - 1 - bi;
            const int b0 = 32 * b, bs = min(32, n - b0);
            for (int base = g.tid; base < 32 * 32; base += 4 * g.nt) {  // four loads in flight
                double v[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int e = base + u * g.nt, r = e >> 5, j = e & 31;
                    v[u] = (e < 32 * 32 && r < bs && j < bs) ? (double)W[(int64_t)s.perm[b0 + r] * n + b0 + j] : 0.0;
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int e = base + u * g.nt;
                    if (e < 32 * 32) blk[(e >> 5) * 33 + (e & 31)] = v[u];
                }
            }
            g.sync();
            for (int q = w; q < kk; q += nw) {
                const int row = b0 + lane;
                const double* tr = blk + lane * 33;
                double yv = lane < bs ? s.y[row * kBMaxK + q] : 0.0;
                if (lower) {
                    for (int j = 0; j < bs; ++j) {
                        const double xj = __shfl_sync(0xffffffffu, yv, j);
                        if (lane > j) yv = (double)((T)yv - (T)tr[j] * (T)xj);
                    }
                } else {
                    for (int j = bs - 1; j >= 0; --j) {
                        if (lane == j) yv = (double)((T)yv / (T)tr[j]);
                        const double xj = __shfl_sync(0xffffffffu, yv, j);
                        if (lane < j) yv = (double)((T)yv - (T)tr[j] * (T)xj);
                    }
                }
                if (lane < bs) s.y[row * kBMaxK + q] = yv;
            }
            g.sync();
            // fold the block into the other rows: a thread per row, every right-hand side (the
            // row of the factor is read once, 8 loads in flight; same order of terms per entry)
            const int rlo = lower ? b0 + bs : 0, rhi = lower ? n : b0;
            for (int r = rlo + g.tid; r < rhi; r += g.nt) {
                const T* lr = W + (int64_t)s.perm[r] * n + b0;
                T acc[kBMaxK];
#pragma unroll
                for (int q = 0; q < kBMaxK; ++q) acc[q] = q < kk ? (T)s.y[r * kBMaxK + q] : (T)0;
#pragma unroll
                for (int j0 = 0; j0 < 32; j0 += 8) {
                    T v[8];
#pragma unroll
                    for (int e2 = 0; e2 < 8; ++e2) v[e2] = j0 + e2 < bs ? lr[j0 + e2] : (T)0;
#pragma unroll
                    for (int e2 = 0; e2 < 8; ++e2) {
                        if (j0 + e2 < bs) {
                            const double* yr = s.y + (b0 + j0 + e2) * kBMaxK;
#pragma unroll
                            for (int q = 0; q < kBMaxK; ++q)
                                if (q < kk) acc[q] -= v[e2] * (T)yr[q];
                        }
                    }
                }
#pragma unroll
                for (int q = 0; q < kBMaxK; ++q)
                    if (q < kk) s.y[r * kBMaxK + q] = (double)acc[q];
            }
            g.sync();
        }
    }
}

// plain FP64 solve of one system
__device__ int solve_plain(const Grp& g, const Slice& s, const BatchArgs& a, int sys, double* W) {
    const int n = a.n[sys], kk = a.k[sys];
    const double* A = a.A + a.a_off[sys];
    if (grp_lu<double>(g, s, A, W, n, s.pw)) return 1;
    const double* B = a.B + a.b_off[sys];
    for (int base = g.tid; base < n * kk; base += 4 * g.nt) {  // four loads in flight
        double v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = base + u * g.nt;
            v[u] = e < n * kk ? B[(int64_t)s.perm[e / kk] * kk + e % kk] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int e = base + u * g.nt;
            if (e < n * kk) s.y[(e / kk) * kBMaxK + e % kk] = v[u];
        }
    }
    g.sync();
    grp_solve<double>(g, s, W, n, kk);
    double* X = a.X + a.b_off[sys];
    for (int e = g.tid; e < n * kk; e += g.nt) {
        const int i = e / kk, q = e - i * kk;
        X[e] = s.y[i * kBMaxK + q];
    }
    g.sync();
    return 0;
}

// FP32 factorisation + FP64 refinement; returns refinement steps, or -1 when FP64 is needed
__device__ int solve_mixed(const Grp& g, const Slice& s, const BatchArgs& a, int sys, double* Wd) {
    const int n = a.n[sys], kk = a.k[sys];
    float* W = reinterpret_cast<float*>(Wd);
    const double* A = a.A + a.a_off[sys];
    const double* B = a.B + a.b_off[sys];
    double* X = a.X + a.b_off[sys];
    if (grp_lu<float>(g, s, A, W, n, s.pw)) return -1;
    // ||A||inf: a warp per row
    const int lane = g.tid & 31, wp = g.tid >> 5, nw = g.nt >> 5;
    double an = 0.0;
    for (int i = wp; i < n; i += nw) {
        double rs = 0.0;
        for (int j = lane; j < n; j += 32) rs += fabs(A[(int64_t)i * n + j]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) rs += __shfl_xor_sync(0xffffffffu, rs, o);
        an = fmax(an, rs);
    }
    double bv;
    int bi;
    grp_argmax(g, s, an, 0, bv, bi);
    const double normA = bv;
    for (int e = g.tid; e < n * kk; e += g.nt) X[e] = 0.0;
    // r = b in factor order
    for (int e = g.tid; e < n * kk; e += g.nt) {
        const int i = e / kk, q = e - i * kk;
        s.y[i * kBMaxK + q] = B[(int64_t)s.perm[i] * kk + q];
    }
    g.sync();
    const double tol = (double)n * 0x1.0p-53;
    const int nmax = s.us - 1;
    double* res = s.pan;  // [n][kBMaxK] residual, natural order (the panel buffer is free now)
    unsigned long long* mx = reinterpret_cast<unsigned long long*>(s.pan + (size_t)nmax * kBMaxK);  // [3][8]
    double prev = INFINITY;
    for (int it = 1; it <= a.max_iter; ++it) {
        grp_solve<float>(g, s, W, n, kk);
        for (int e = g.tid; e < n * kk; e += g.nt) {
            const int i = e / kk, q = e - i * kk;
            const double xv = X[e] + s.y[i * kBMaxK + q];
            X[e] = xv;
            s.y[i * kBMaxK + q] = xv;  // x in natural order for the residual below
        }
        if (g.tid < 3 * kBMaxK) mx[g.tid] = 0ull;
        g.sync();
        // r = b - A x in FP64, a warp per row (coalesced rows of A), with the column maxima
        for (int i = wp; i < n; i += nw) {
            double acc[kBMaxK];
#pragma unroll
            for (int q = 0; q < kBMaxK; ++q) acc[q] = 0.0;
            for (int j = lane; j < n; j += 32) {
                const double aij = A[(int64_t)i * n + j];
#pragma unroll
                for (int q = 0; q < kBMaxK; ++q)
                    if (q < kk) acc[q] = fma(aij, s.y[j * kBMaxK + q], acc[q]);
            }
#pragma unroll
            for (int q = 0; q < kBMaxK; ++q) {
                double v = acc[q];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if (lane == q && q < kk) {
                    const double bq = B[(int64_t)i * kk + q], xq = s.y[i * kBMaxK + q];
                    const double rq = bq - v;
                    res[i * kBMaxK + q] = rq;
                    atomicMax(&mx[q], (unsigned long long)__double_as_longlong(fabs(rq)));
                    atomicMax(&mx[kBMaxK + q], (unsigned long long)__double_as_longlong(fabs(xq)));
                    atomicMax(&mx[2 * kBMaxK + q], (unsigned long long)__double_as_longlong(fabs(bq)));
                }
            }
        }
        g.sync();
        double eta = 0.0;
        for (int q = 0; q < kk; ++q) {
            const double r1 = __longlong_as_double((long long)mx[q]);
            const double x1 = __longlong_as_double((long long)mx[kBMaxK + q]);
            const double b1 = __longlong_as_double((long long)mx[2 * kBMaxK + q]);
            const double den = normA * x1 + b1;
            eta = fmax(eta, den > 0.0 ? r1 / den : (r1 > 0.0 ? INFINITY : 0.0));
        }
        for (int e = g.tid; e < n * kk; e += g.nt) {
            const int i = e / kk, q = e - i * kk;
            s.y[i * kBMaxK + q] = res[s.perm[i] * kBMaxK + q];
        }
        g.sync();
        if (eta <= tol) return it;
        if (!(eta < INFINITY) || (it >= 2 && eta > 0.5 * prev)) return -1;
        prev = eta;
    }
    return -1;
}

// MODE 0 plain FP64, 1 FP32 factor + FP64 refinement.  At most 128 registers a thread, so that
// two CTAs share an SM whenever the tile shape's shared memory allows it.
template <int MODE>
__global__ void __launch_bounds__(kBThreads, 2) batch_solve_kernel(BatchArgs a) {
    extern __shared__ __align__(16) double bsm[];
    __shared__ int s_sys[8];
    const int t = threadIdx.x;
    double* W = a.scratch + (size_t)blockIdx.x * batch_scratch_doubles(a.small_n, a.group_warps, a.big_warps);
    for (;;) {
        if (t == 0) s_sys[0] = atomicAdd(a.counter, 1);
        __syncthreads();
        const int idx = s_sys[0];
        __syncthreads();
        if (idx >= a.count) return;
        // this system and up to ng - 1 more from the queue, one per group; the first one decides
        // the round's group size and slice shape (the queue is sorted largest first, so a round
        // that starts with a large system may end with small ones, which fit its slices too)
        const bool big = a.n[a.order[idx]] > a.small_n;
        const int gw = big ? a.big_warps : a.group_warps, ng = (kBThreads / 32) / gw;
        const int nmax = big ? kBMaxN : a.small_n, pw = big ? a.pw_large : a.pw_small;
        if (t == 0) {
            for (int q = 1; q < ng; ++q) {
                const int j = atomicAdd(a.counter, 1);
                s_sys[q] = j < a.count ? j : -1;
            }
        }
        __syncthreads();
        const int gi = t / (32 * gw);
        const int myidx = s_sys[gi];
        if (myidx >= 0) {
            const int msys = a.order[myidx];
            const Grp g{t - gi * 32 * gw, 32 * gw, 2 + gi};
            const Slice s = carve(bsm + (size_t)gi * slice_doubles(nmax, pw), nmax, pw);
            double* Wg = W + (size_t)gi * nmax * nmax;
            int st, iters = 0;
            if (MODE == 1) {
                iters = solve_mixed(g, s, a, msys, Wg);
                st = iters < 0 ? solve_plain(g, s, a, msys, Wg) : 0;
            } else {
                st = solve_plain(g, s, a, msys, Wg);
            }
            if (g.tid == 0) {
                a.info[msys] = st;
                if (a.iters) a.iters[msys] = iters;
            }
        }
        __syncthreads();
    }
}

size_t batch_smem_bytes(int small_n, int G, int pw_large, int pw_small, int GB) {
    const size_t big = slice_doubles(kBMaxN, pw_large) * ((kBThreads / 32) / GB);
    const size_t small = slice_doubles(small_n, pw_small) * ((kBThreads / 32) / G);
    return std::max(big, small) * sizeof(double);
}

}  // namespace

// ------------------------------------------------------------------ host side
struct BatchPlanCache {
    std::vector<int32_t> n, k;
    std::vector<int64_t> a_off, b_off;
    int64_t count = -1;
};

int32_t batch_solve(Ctx* ctx, cudaStream_t st, int64_t count, const int32_t* hn, const int32_t* hk,
                    const int64_t* ha_off, const int64_t* hb_off, const double* A, const double* B, double* X,
                    int mode, int32_t* info, int32_t* iters, BatchTune* tune_out) {
    if (count <= 0) return B2M_OK;
    if (mode != 0 && mode != 1) return fail(ctx, B2M_ERR_ARG, "batch: mode must be 0 (FP64) or 1 (FP32 + FP64 IR)");
    for (int64_t i = 0; i < count; ++i) {
        if (hn[i] < 1 || hn[i] > kBMaxN) return fail(ctx, B2M_ERR_UNSUPPORTED, "batch: system %lld order %d not in [1, 256]", (long long)i, hn[i]);
        if (hk[i] < 1 || hk[i] > kBMaxK) return fail(ctx, B2M_ERR_UNSUPPORTED, "batch: system %lld has %d right-hand sides (1..8)", (long long)i, hk[i]);
    }
    // device copies of the plan: n, k, offsets, order (largest first), queue head
    std::vector<int32_t> order((size_t)count);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) { return hn[x] > hn[y]; });
    const size_t bytes_i = (size_t)count * 4, bytes_l = (size_t)count * 8;
    const size_t plan_bytes = 3 * bytes_i + 2 * bytes_l + 256;
    void* pplan;
    B2M_TRY(ws_get(ctx, kWsH, plan_bytes + 256, &pplan));
    char* pp = static_cast<char*>(pplan);
    int32_t* dn = reinterpret_cast<int32_t*>(pp);
    int32_t* dk = dn + count;
    int32_t* dord = dk + count;
    int64_t* dao = reinterpret_cast<int64_t*>(pp + round_up((int64_t)(3 * bytes_i), 256));
    int64_t* dbo = dao + count;
    int32_t* dctr = reinterpret_cast<int32_t*>(dbo + count);
    uint64_t sig = 1469598103934665603ull ^ (uint64_t)mode;
    for (int64_t i = 0; i < count; ++i)
        sig = (sig ^ (uint64_t)(hn[i] * 16 + hk[i]) ^ ((uint64_t)ha_off[i] << 20) ^ ((uint64_t)hb_off[i] << 40)) *
              1099511628211ull;
    const bool same_plan = ctx->batch_plan_sig == sig && ctx->batch_plan_dev == pplan;
    void* ph = nullptr;
    if (!same_plan) {
        // the pinned staging buffer may still feed an earlier asynchronous copy
        B2M_CU(ctx, cudaStreamSynchronize(st));
        B2M_TRY(pinned_get(ctx, plan_bytes + 256, &ph));
    }
    if (!same_plan) {
        char* hp = static_cast<char*>(ph);
        std::memcpy(hp, hn, bytes_i);
        std::memcpy(hp + bytes_i, hk, bytes_i);
        std::memcpy(hp + 2 * bytes_i, order.data(), bytes_i);
        std::memcpy(hp + round_up((int64_t)(3 * bytes_i), 256), ha_off, bytes_l);
        std::memcpy(hp + round_up((int64_t)(3 * bytes_i), 256) + bytes_l, hb_off, bytes_l);
        B2M_CU(ctx, cudaMemcpyAsync(pp, hp, round_up((int64_t)(3 * bytes_i), 256) + 2 * bytes_l,
                                    cudaMemcpyHostToDevice, st));
        ctx->batch_plan_sig = sig;
        ctx->batch_plan_dev = pplan;
    }

    int occ_sms = ctx->num_sms;
    BatchArgs a{};
    a.count = (int)count;
    a.n = dn; a.k = dk; a.a_off = dao; a.b_off = dbo;
    a.A = A; a.B = B; a.X = X;
    a.order = dord; a.counter = dctr; a.info = info; a.iters = iters;
    a.mode = mode;
    a.max_iter = 10;

    auto launch = [&](const BatchTune& tc, cudaStream_t q) -> int32_t {
        const size_t smem = batch_smem_bytes(tc.small_n, tc.group_warps, tc.pw_large, tc.pw_small, tc.big_warps);
        void (*kern)(BatchArgs) = mode == 1 ? batch_solve_kernel<1> : batch_solve_kernel<0>;
        B2M_CU(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0;
        B2M_CU(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBThreads, smem));
        if (per_sm < 1) return fail(ctx, B2M_ERR_UNSUPPORTED, "batch: tile shape does not fit one SM");
        const int grid = occ_sms * per_sm;
        void* pscr;
        B2M_TRY(ws_get(ctx, kWsMatD,
                       (size_t)grid * batch_scratch_doubles(tc.small_n, tc.group_warps, tc.big_warps) * sizeof(double),
                       &pscr));
        BatchArgs b = a;
        b.scratch = static_cast<double*>(pscr);
        b.small_n = tc.small_n;
        b.group_warps = tc.group_warps;
        b.big_warps = tc.big_warps;
        b.pw_large = tc.pw_large;
        b.pw_small = tc.pw_small;
        B2M_CU(ctx, cudaMemsetAsync(dctr, 0, sizeof(int32_t), q));
        prof_begin(ctx, q, kClsSolve);
        kern<<<grid, kBThreads, smem, q>>>(b);
        prof_end(ctx, q, kClsSolve, 0.0);
        B2M_LAUNCHED(ctx);
        return B2M_OK;
    };

    // autotune once per plan (mode, sizes, layout): time each candidate shape on this batch
    BatchTune best;
    auto it = ctx->batch_tunes.find(sig);
    if (it != ctx->batch_tunes.end()) {
        best = it->second;
    } else {
        std::vector<BatchTune> cands;
        for (int GB : {8, 4})
            for (int pwl : {8, 16, 32})
                for (int G : {1, 2, 4})
                    for (int pws : {8, 16}) cands.push_back(BatchTune{64, G, pwl, pws, GB, 0.0f});
        cudaEvent_t e0, e1;
        B2M_CU(ctx, cudaEventCreate(&e0));
        B2M_CU(ctx, cudaEventCreate(&e1));
        float best_ms = 1e30f;
        for (auto& c : cands) {
            const size_t smem = batch_smem_bytes(c.small_n, c.group_warps, c.pw_large, c.pw_small, c.big_warps);
            if (smem > ctx->smem_optin) continue;
            B2M_TRY(launch(c, st));  // warm
            B2M_CU(ctx, cudaEventRecord(e0, st));
            B2M_TRY(launch(c, st));
            B2M_CU(ctx, cudaEventRecord(e1, st));
            B2M_CU(ctx, cudaEventSynchronize(e1));
            float ms = 0.f;
            B2M_CU(ctx, cudaEventElapsedTime(&ms, e0, e1));
            c.ms = ms;
            if (ms < best_ms) { best_ms = ms; best = c; }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (best_ms >= 1e30f) return fail(ctx, B2M_ERR_UNSUPPORTED, "batch: no tile shape fits");
        ctx->batch_tunes[sig] = best;
    }
    if (tune_out) *tune_out = best;
    const GraphKey key{7 + mode * 10, A, B, X, info, count, (int64_t)sig,
                       best.big_warps * 1000000 + best.pw_large * 10000 + best.pw_small * 100 + best.group_warps,
                       (int64_t)reinterpret_cast<intptr_t>(iters)};
    return run_graph(ctx, st, key, [&](cudaStream_t q) { return launch(best, q); });
}

}  // namespace b2m

// ------------------------------------------------------------------ persisted autotuner table
// One text line per batch plan: "<plan signature, hex> <small_n> <group_warps> <pw_large> <pw_small>
// <big_warps> <ms>", after the header line "b2m-batch-tune 2" (a version-1 table, without the
// big_warps column, is read as big_warps = 8).  A later process that loads the table skips the
// timing of the candidate shapes for every plan it lists (the signature covers the mode, every
// system's order, right-hand sides and offsets).
extern "C" int32_t b2m_batch_tune_save(b2m_ctx* h, const char* path) {
    b2m::Ctx* ctx = reinterpret_cast<b2m::Ctx*>(h);
    if (!ctx || !path) return B2M_ERR_ARG;
    b2m::CallLock lk(ctx);
    FILE* f = std::fopen(path, "w");
    if (!f) return b2m::fail(ctx, B2M_ERR_ARG, "cannot write %s", path);
    std::fprintf(f, "b2m-batch-tune 2\n");
    for (const auto& e : ctx->batch_tunes)
        std::fprintf(f, "%016llx %d %d %d %d %d %.6f\n", (unsigned long long)e.first, e.second.small_n,
                     e.second.group_warps, e.second.pw_large, e.second.pw_small, e.second.big_warps,
                     (double)e.second.ms);
    return std::fclose(f) == 0 ? B2M_OK : b2m::fail(ctx, B2M_ERR_ARG, "cannot write %s", path);
}

extern "C" int32_t b2m_batch_tune_load(b2m_ctx* h, const char* path, int32_t* loaded) {
    b2m::Ctx* ctx = reinterpret_cast<b2m::Ctx*>(h);
    if (!ctx || !path) return B2M_ERR_ARG;
    b2m::CallLock lk(ctx);
    if (loaded) *loaded = 0;
    FILE* f = std::fopen(path, "r");
    if (!f) return b2m::fail(ctx, B2M_ERR_ARG, "cannot read %s", path);
    char head[32] = {0};
    int version = 0;
    if (std::fscanf(f, "%31s %d", head, &version) != 2 || std::strcmp(head, "b2m-batch-tune") != 0 ||
        (version != 1 && version != 2)) {
        std::fclose(f);
        return b2m::fail(ctx, B2M_ERR_FORMAT, "%s is not a batch tuning table", path);
    }
    unsigned long long sig;
    int sn, g, pwl, pws, gb = 8;
    double ms;
    int n = 0;
    auto next = [&]() -> bool {
        if (version == 1) return std::fscanf(f, "%llx %d %d %d %d %lf", &sig, &sn, &g, &pwl, &pws, &ms) == 6;
        return std::fscanf(f, "%llx %d %d %d %d %d %lf", &sig, &sn, &g, &pwl, &pws, &gb, &ms) == 7;
    };
    while (next()) {
        // only shapes the kernel has: a damaged or foreign line is skipped, never launched
        const bool ok = sn == 64 && (g == 1 || g == 2 || g == 4) && (pwl == 8 || pwl == 16 || pwl == 32) &&
                        (pws == 8 || pws == 16) && (gb == 4 || gb == 8) &&
                        b2m::batch_smem_bytes(sn, g, pwl, pws, gb) <= ctx->smem_optin;
        if (!ok) continue;
        ctx->batch_tunes[(uint64_t)sig] = b2m::BatchTune{sn, g, pwl, pws, gb, (float)ms};
        ++n;
    }
    std::fclose(f);
    if (loaded) *loaded = n;
    return B2M_OK;
}
