// mrmath_oracle.cpp -- CPU restatement of mrMath's dense FP64 GEMM + pivoted-LU path.
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA product and the timed CPU baseline.
// The product (libb2m) never links or calls this file.
//
// Compiled with -ffp-contract=off so that every multiply/add is rounded exactly where the
// reference rounds it; fused multiply-adds appear only where the reference's FMA kernels
// issue vfmadd231pd (FMAMatrixMultTransposedOperationsx64.pas), written as std::fma or
// _mm256_fmadd_pd.
#include "mrmath_oracle.h"

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>
#include <unistd.h>
#include <immintrin.h>

namespace {

inline double* rowp(double* A, int64_t r, int64_t lw) { return (double*)((char*)A + r * lw); }
inline const double* rowp(const double* A, int64_t r, int64_t lw) {
    return (const double*)((const char*)A + r * lw);
}

int g_mode = 1;  // itFMA is the dispatch default (MatrixASMStubSwitch.pas:2080-2084)

// ------------------------------------------------------------------------------------
// random engine
// ------------------------------------------------------------------------------------
const int kN = 624, kM = 397;
const uint32_t kMatrixA = 0x9908b0dfu, kUpper = 0x80000000u, kLower = 0x7fffffffu;

}  // namespace

extern "C" void orc_rng_init(orc_rng* r, int32_t seed) {
    // InitMersenne RandomEng.pas:626-644 (seed 0 would mean "time"; callers pass a seed)
    r->mt[0] = (uint32_t)seed;
    for (uint32_t i = 1; i < (uint32_t)kN; ++i)
        r->mt[i] = 1812433253u * (r->mt[i - 1] ^ (r->mt[i - 1] >> 30)) + i;
    r->mti = kN;
    r->gauss_flag = 0;
    r->gauss2 = 0.0;
}

extern "C" void orc_rng_init_by_array(orc_rng* r, const uint32_t* key, int32_t len) {
    // InitMersenneByArr RandomEng.pas:646-692
    orc_rng_init(r, 19650218);
    uint32_t i = 1, j = 0;
    for (int k = std::max(kN, (int)len) - 1; k >= 0; --k) {
        r->mt[i] = (r->mt[i] ^ ((r->mt[i - 1] ^ (r->mt[i - 1] >> 30)) * 1664525u)) + key[j] + j;
        ++i; ++j;
        if (i >= (uint32_t)kN) { r->mt[0] = r->mt[kN - 1]; i = 1; }
        if (j > (uint32_t)(len - 1)) j = 0;
    }
    for (int k = kN - 2; k >= 0; --k) {
        r->mt[i] = (r->mt[i] ^ ((r->mt[i - 1] ^ (r->mt[i - 1] >> 30)) * 1566083941u)) - i;
        ++i;
        if (i >= (uint32_t)kN) { r->mt[0] = r->mt[kN - 1]; i = 1; }
    }
    r->mt[0] = 0x80000000u;
}

extern "C" uint32_t orc_rng_u32(orc_rng* r) {
    // RandMersenneDblWord RandomEng.pas:694-731
    static const uint32_t mag01[2] = {0u, kMatrixA};
    if (r->mti > kN) orc_rng_init(r, 5489);
    if (r->mti >= kN) {
        int kk;
        uint32_t y;
        for (kk = 0; kk < kN - kM; ++kk) {
            y = (r->mt[kk] & kUpper) | (r->mt[kk + 1] & kLower);
            r->mt[kk] = r->mt[kk + kM] ^ (y >> 1) ^ mag01[y & 1u];
        }
        for (; kk < kN - 1; ++kk) {
            y = (r->mt[kk] & kUpper) | (r->mt[kk + 1] & kLower);
            r->mt[kk] = r->mt[kk + (kM - kN)] ^ (y >> 1) ^ mag01[y & 1u];
        }
        y = (r->mt[kN - 1] & kUpper) | (r->mt[0] & kLower);
        r->mt[kN - 1] = r->mt[kM - 1] ^ (y >> 1) ^ mag01[y & 1u];
        r->mti = 0;
    }
    uint32_t y = r->mt[r->mti++];
    y ^= (y >> 11);
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= (y >> 18);
    return y;
}

extern "C" uint32_t orc_rng_lw(orc_rng* r, uint32_t range) { return orc_rng_u32(r) % range; }

extern "C" double orc_rng_dbl(orc_rng* r) {
    // RandMersenneDbl RandomEng.pas:749-765: (a>>5 * 2^26 + b>>6) * 2^-53
    const double multA = 67108864.0, multB = 1.0 / 9007199254740992.0;
    uint32_t a = orc_rng_u32(r);
    double x = (double)(a >> 5);
    uint32_t b = orc_rng_u32(r);
    double y = (double)(b >> 6);
    return (x * multA + y) * multB;
}

extern "C" double orc_rng_gauss(orc_rng* r) {
    // RandGauss RandomEng.pas:283-307 (Marsaglia polar method, two values per round)
    double res;
    if (r->gauss_flag) {
        res = r->gauss2;
    } else {
        double v1, v2, rsq;
        do {
            v1 = 2.0 * orc_rng_dbl(r) - 1.0;
            v2 = 2.0 * orc_rng_dbl(r) - 1.0;
            rsq = v1 * v1 + v2 * v2;
        } while (!(rsq < 1.0 && rsq != 0.0));
        res = std::sqrt(-2.0 * std::log(rsq) / rsq);
        r->gauss2 = v1 * res;
        res = v2 * res;
    }
    r->gauss_flag = !r->gauss_flag;
    return res;
}

extern "C" void orc_fill_uniform(orc_rng* r, double* dst, int64_t count) {
    for (int64_t i = 0; i < count; ++i) dst[i] = orc_rng_dbl(r);
}
extern "C" void orc_fill_gauss(orc_rng* r, double* dst, int64_t count) {
    for (int64_t i = 0; i < count; ++i) dst[i] = orc_rng_gauss(r);
}
extern "C" void orc_fill_gauss_exp(orc_rng* r, double* dst, int64_t count) {
    // all Gaussians first, then all exponents e = RandLW(17) - 8, applied element by element
    for (int64_t i = 0; i < count; ++i) dst[i] = orc_rng_gauss(r);
    for (int64_t i = 0; i < count; ++i) dst[i] = std::ldexp(dst[i], (int)orc_rng_lw(r, 17u) - 8);
}

extern "C" void orc_set_mode(int32_t mode) { g_mode = mode ? 1 : 0; }
extern "C" int32_t orc_get_mode(void) { return g_mode; }

namespace {

// ------------------------------------------------------------------------------------
// element kernels (SimpleMatrixOperations.pas; the AVX versions compute the same values)
// ------------------------------------------------------------------------------------
void mtx_copy(double* dest, int64_t lwd, const double* src, int64_t lws, int64_t w, int64_t h) {
    for (int64_t y = 0; y < h; ++y) std::memcpy(rowp(dest, y, lwd), rowp(src, y, lws), w * sizeof(double));
}
void mtx_add(double* dest, int64_t lwd, const double* m1, const double* m2, int64_t w, int64_t h,
             int64_t lw1, int64_t lw2) {
    for (int64_t y = 0; y < h; ++y) {
        double* d = rowp(dest, y, lwd);
        const double* a = rowp(m1, y, lw1);
        const double* b = rowp(m2, y, lw2);
        for (int64_t x = 0; x < w; ++x) d[x] = a[x] + b[x];
    }
}
void mtx_sub(double* dest, int64_t lwd, const double* m1, const double* m2, int64_t w, int64_t h,
             int64_t lw1, int64_t lw2) {
    // GenericMtxSub SimpleMatrixOperations.pas:1380-1394
    for (int64_t y = 0; y < h; ++y) {
        double* d = rowp(dest, y, lwd);
        const double* a = rowp(m1, y, lw1);
        const double* b = rowp(m2, y, lw2);
        for (int64_t x = 0; x < w; ++x) d[x] = a[x] - b[x];
    }
}
void mtx_transpose(double* dest, int64_t lwd, const double* src, int64_t lws, int64_t w, int64_t h) {
    // dest (w x h) = src(h x w)^T
    for (int64_t y = 0; y < h; ++y) {
        const double* s = rowp(src, y, lws);
        for (int64_t x = 0; x < w; ++x) rowp(dest, x, lwd)[y] = s[x];
    }
}
void row_swap(double* a, double* b, int64_t w) {
    // GenericRowSwap SimpleMatrixOperations.pas:1013-1026
    for (int64_t i = 0; i < w; ++i) std::swap(a[i], b[i]);
}

// GenericMtxMult SimpleMatrixOperations.pas:1561-1591: dest := dest + a*b from 0, sequential k.
void generic_mult(double* dest, int64_t lwd, const double* mt1, const double* mt2, int64_t w1, int64_t h1,
                  int64_t w2, int64_t /*h2*/, int64_t lw1, int64_t lw2) {
    for (int64_t y = 0; y < h1; ++y) {
        const double* a = rowp(mt1, y, lw1);
        double* d = rowp(dest, y, lwd);
        for (int64_t x = 0; x < w2; ++x) {
            double s = 0.0;
            for (int64_t k = 0; k < w1; ++k) s = s + a[k] * rowp(mt2, k, lw2)[x];
            d[x] = s;
        }
    }
}
// GenericMtxMultTransp SimpleMatrixOperations.pas:1593-1617: dest(h1 x h2) = mt1 * mt2^T
void generic_mult_transp(double* dest, int64_t lwd, const double* mt1, const double* mt2, int64_t w1,
                         int64_t h1, int64_t /*w2*/, int64_t h2, int64_t lw1, int64_t lw2) {
    for (int64_t y = 0; y < h1; ++y) {
        const double* a = rowp(mt1, y, lw1);
        double* d = rowp(dest, y, lwd);
        for (int64_t x = 0; x < h2; ++x) {
            const double* b = rowp(mt2, x, lw2);
            double s = 0.0;
            for (int64_t k = 0; k < w1; ++k) s = s + a[k] * b[k];
            d[x] = s;
        }
    }
}

// The FMA kernel's per-entry summation order (FMAMatrixMultTransposedOperationsx64.pas:593-760,
// and the Mod16 variants :40-375): four lanes l0..l3 accumulate k = 4q + lane with vfmadd231pd,
// then vhaddpd gives (l0+l1, l2+l3); the k mod 4 tail is added to (l0+l1) with separate
// vmulsd/vaddsd; the final vhaddpd returns (l0+l1+tail) + (l2+l3).
inline double dot_fma4_scalar(const double* a, const double* b, int64_t K) {
    double l0 = 0.0, l1 = 0.0, l2 = 0.0, l3 = 0.0;
    const int64_t g = K / 4;
    for (int64_t q = 0; q < g; ++q) {
        l0 = std::fma(a[4 * q + 0], b[4 * q + 0], l0);
        l1 = std::fma(a[4 * q + 1], b[4 * q + 1], l1);
        l2 = std::fma(a[4 * q + 2], b[4 * q + 2], l2);
        l3 = std::fma(a[4 * q + 3], b[4 * q + 3], l3);
    }
    double s = 0.0, t = 0.0;
    if (g > 0) { s = l0 + l1; t = l2 + l3; }
    for (int64_t r = 4 * g; r < K; ++r) { double p = a[r] * b[r]; s = s + p; }
    return s + t;
}

__attribute__((target("avx2,fma"))) void multT2_fma_avx2(double* dest, int64_t lwd, const double* mt1,
                                                          const double* mt2, int64_t K, int64_t h1,
                                                          int64_t h2, int64_t lw1, int64_t lw2) {
    // Two outputs per pass as the assembler does (ymm0/ymm2 accumulators); numerics per entry as
    // dot_fma4_scalar.
    const int64_t g = K / 4;
    for (int64_t y = 0; y < h1; ++y) {
        const double* a = rowp(mt1, y, lw1);
        double* d = rowp(dest, y, lwd);
        int64_t x = 0;
        for (; x + 1 < h2; x += 2) {
            const double* b0 = rowp(mt2, x, lw2);
            const double* b1 = rowp(mt2, x + 1, lw2);
            __m256d acc0 = _mm256_setzero_pd(), acc1 = _mm256_setzero_pd();
            for (int64_t q = 0; q < g; ++q) {
                __m256d va = _mm256_loadu_pd(a + 4 * q);
                acc0 = _mm256_fmadd_pd(va, _mm256_loadu_pd(b0 + 4 * q), acc0);
                acc1 = _mm256_fmadd_pd(va, _mm256_loadu_pd(b1 + 4 * q), acc1);
            }
            double l0[4], l1[4];
            _mm256_storeu_pd(l0, acc0);
            _mm256_storeu_pd(l1, acc1);
            double s0 = 0.0, t0 = 0.0, s1 = 0.0, t1 = 0.0;
            if (g > 0) { s0 = l0[0] + l0[1]; t0 = l0[2] + l0[3]; s1 = l1[0] + l1[1]; t1 = l1[2] + l1[3]; }
            for (int64_t r = 4 * g; r < K; ++r) {
                double p0 = a[r] * b0[r], p1 = a[r] * b1[r];
                s0 = s0 + p0; s1 = s1 + p1;
            }
            d[x] = s0 + t0;
            d[x + 1] = s1 + t1;
        }
        for (; x < h2; ++x) d[x] = dot_fma4_scalar(a, rowp(mt2, x, lw2), K);
    }
}

bool have_avx2() {
    static int cached = -1;
    if (cached < 0) cached = (__builtin_cpu_supports("avx2") && __builtin_cpu_supports("fma")) ? 1 : 0;
    return cached == 1;
}

// MatrixMultT2 = FMAMatrixMultTransposed (FMAMatrixOperations.pas:55-92) in fma mode,
// GenericMtxMultTransp in generic mode.  dest(h1 x h2) = mt1(h1 x K) * mt2(h2 x K)^T
void matrix_multT2(double* dest, int64_t lwd, const double* mt1, const double* mt2, int64_t K, int64_t h1,
                   int64_t h2, int64_t lw1, int64_t lw2) {
    if (K == 0 || h1 == 0 || h2 == 0) return;
    if (g_mode == 0 || K < 2 || K == 2) {
        // K == 2 goes to the SSE kernel, whose (a0*b0)+(a1*b1) equals the generic order
        generic_mult_transp(dest, lwd, mt1, mt2, K, h1, K, h2, lw1, lw2);
        return;
    }
    if (have_avx2()) {
        multT2_fma_avx2(dest, lwd, mt1, mt2, K, h1, h2, lw1, lw2);
    } else {
        for (int64_t y = 0; y < h1; ++y)
            for (int64_t x = 0; x < h2; ++x)
                rowp(dest, y, lwd)[x] = dot_fma4_scalar(rowp(mt1, y, lw1), rowp(mt2, x, lw2), K);
    }
}

// multFunc = FMAMatrixMult (FMAMatrixOperations.pas:94-148) in fma mode: transpose mt2, then
// FMAMatrixMultTransposed.  Matrix-vector cases use the generic order.
void mult_direct(double* dest, int64_t lwd, const double* mt1, const double* mt2, int64_t w1, int64_t h1,
                 int64_t w2, int64_t h2, int64_t lw1, int64_t lw2) {
    if (w1 == 0 || w2 == 0 || h1 == 0 || h2 == 0) return;
    if (g_mode == 0 || w1 < 2 || w2 < 2) {
        generic_mult(dest, lwd, mt1, mt2, w1, h1, w2, h2, lw1, lw2);
        return;
    }
    int64_t tlw = h2;
    if (tlw & 3) tlw += 4 - (tlw & 3);
    std::vector<double> t((size_t)(w2 * tlw));
    mtx_transpose(t.data(), tlw * 8, mt2, lw2, w2, h2);
    matrix_multT2(dest, lwd, mt1, t.data(), w1, h1, w2, lw1, tlw * 8);
}

int64_t next2pwr(int64_t num, int64_t maxSize) {
    int64_t r = 1;
    while (r < maxSize && r < num) r <<= 1;
    return r;
}

// BlockMatrixMultiplication BlockedMult.pas:350-474.  Output rows [y0, y1) only, so the
// threaded twins can split the same computation without changing any value.
void block_mult_rows(double* dest, int64_t lwd, const double* mt1, const double* mt2, int64_t w1, int64_t h1,
                     int64_t w2, int64_t /*h2*/, int64_t lw1, int64_t lw2, int64_t bs, int32_t op,
                     int64_t bx0, int64_t bx1) {
    const bool h1Fit = (h1 % bs) == 0, w2Fit = (w2 % bs) == 0, w1Fit = (w1 % bs) == 0;
    const int64_t h = h1 / bs + (h1Fit ? 0 : 1) - 1;
    const int64_t w = w2 / bs + (w2Fit ? 0 : 1) - 1;
    const int64_t gamma = w1 / bs + (w1Fit ? 0 : 1) - 1;
    std::vector<double> actBlk((size_t)(bs * bs)), multBlk((size_t)(bs * bs)), transBlk((size_t)(bs * bs));
    const int64_t bl = bs * 8;
    for (int64_t by = 0; by <= h; ++by) {
        const int64_t blkHeight = (by == h && !h1Fit) ? h1 % bs : bs;
        const double* pA0 = rowp(mt1, by * bs, lw1);
        for (int64_t bx = bx0; bx <= std::min(w, bx1 - 1); ++bx) {
            const int64_t blkWidth = (bx == w && !w2Fit) ? w2 % bs : bs;
            std::fill(actBlk.begin(), actBlk.end(), 0.0);
            const double* pa = pA0;
            const double* pb = mt2 + bx * bs;
            for (int64_t idx = 0; idx <= gamma; ++idx) {
                const int64_t gw = (idx == gamma && !w1Fit) ? w1 % bs : bs;
                if (blkWidth > 3 && blkHeight > 3) {
                    mtx_transpose(transBlk.data(), bl, pb, lw2, blkWidth, gw);
                    matrix_multT2(multBlk.data(), bl, pa, transBlk.data(), gw, blkHeight, blkWidth, lw1, bl);
                } else {
                    generic_mult(multBlk.data(), bl, pa, pb, gw, blkHeight, blkWidth, gw, lw1, lw2);
                }
                mtx_add(actBlk.data(), bl, actBlk.data(), multBlk.data(), blkWidth, blkHeight, bl, bl);
                pa += gw;
                pb = rowp(pb, gw, lw2);
            }
            double* pDest = rowp(dest, by * bs, lwd) + bx * bs;
            if (op == 0) mtx_copy(pDest, lwd, actBlk.data(), bl, blkWidth, blkHeight);
            else if (op == 1) mtx_add(pDest, lwd, pDest, actBlk.data(), blkWidth, blkHeight, lwd, bl);
            else mtx_sub(pDest, lwd, pDest, actBlk.data(), blkWidth, blkHeight, lwd, bl);
        }
    }
}

void block_mult(double* dest, int64_t lwd, const double* mt1, const double* mt2, int64_t w1, int64_t h1,
                int64_t w2, int64_t h2, int64_t lw1, int64_t lw2, int64_t bs, int32_t op, bool haveMem) {
    if (w1 == 0 || w2 == 0 || h1 == 0 || h2 == 0) return;
    if (bs > w1 && !haveMem) bs = next2pwr(w1, bs);
    block_mult_rows(dest, lwd, mt1, mt2, w1, h1, w2, h2, lw1, lw2, bs, op, 0, INT64_MAX / 2);
}

// MatrixMult MatrixASMStubSwitch.pas:769-776 (BlockedMatrixMultSize = 512, BlockMatrixCacheSize = 128)
void matrix_mult(double* dest, int64_t lwd, const double* mt1, const double* mt2, int64_t w1, int64_t h1,
                 int64_t w2, int64_t h2, int64_t lw1, int64_t lw2) {
    if (w1 >= 512 && h1 >= 512 && h2 >= 512 && w2 >= 512)
        block_mult(dest, lwd, mt1, mt2, w1, h1, w2, h2, lw1, lw2, 128, 0, false);
    else
        mult_direct(dest, lwd, mt1, mt2, w1, h1, w2, h2, lw1, lw2);
}

// ------------------------------------------------------------------------------------
// thread pool standing in for MtxThreadPool (task group = AddTaskRec + SyncAll; the caller
// runs the last task itself, as every threaded routine of the reference does)
// ------------------------------------------------------------------------------------
class Pool {
  public:
    explicit Pool(int n) { resize(n); }
    ~Pool() { stop(); }
    void resize(int n) {
        stop();
        quit_ = false;
        for (int i = 0; i < n - 1; ++i) workers_.emplace_back([this] { loop(); });
        n_ = n;
    }
    int size() const { return n_; }
    void run(std::vector<std::function<void()>>& tasks) {
        if (tasks.empty()) return;
        std::atomic<int> left((int)tasks.size() - 1);
        {
            std::lock_guard<std::mutex> lk(m_);
            for (size_t i = 0; i + 1 < tasks.size(); ++i)
                q_.push_back([&tasks, i, &left] { tasks[i](); left.fetch_sub(1); });
        }
        cv_.notify_all();
        tasks.back()();
        // SyncAll: help with queued work, then wait
        for (;;) {
            std::function<void()> f;
            {
                std::lock_guard<std::mutex> lk(m_);
                if (!q_.empty()) { f = std::move(q_.back()); q_.pop_back(); }
            }
            if (f) { f(); continue; }
            if (left.load() == 0) break;
            std::this_thread::yield();
        }
    }

  private:
    void loop() {
        for (;;) {
            std::function<void()> f;
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [this] { return quit_ || !q_.empty(); });
                if (quit_ && q_.empty()) return;
                f = std::move(q_.front());
                q_.erase(q_.begin());
            }
            f();
        }
    }
    void stop() {
        {
            std::lock_guard<std::mutex> lk(m_);
            quit_ = true;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
        workers_.clear();
    }
    std::vector<std::thread> workers_;
    std::vector<std::function<void()>> q_;
    std::mutex m_;
    std::condition_variable cv_;
    bool quit_ = false;
    int n_ = 1;
};

int g_threads = 0;
Pool* pool() {
    static Pool* p = nullptr;
    if (!p) {
        if (g_threads <= 0) g_threads = std::max(1L, sysconf(_SC_NPROCESSORS_ONLN));  // linuxthrpool.pas:265
        g_threads = std::min(g_threads, 64);  // cMaxNumCores MtxThreadPool.pas:68
        p = new Pool(g_threads);
    }
    return p;
}

// NumCoresToUseForMult ThreadedMatrixOperations.pas:486-503
int num_cores_for_mult(int64_t w1, int64_t h1, int64_t w2, int64_t /*h2*/, int64_t bs) {
    const int nc = pool()->size();
    if (w1 <= bs && w2 <= bs) {
        int r = 1;
        if (h1 > bs) r = (int)std::min<int64_t>(nc, 1 + h1 / bs);
        return r;
    }
    int64_t numBlocks = h1 / bs + w2 / bs;
    return (int)std::max<int64_t>(1, std::min<int64_t>(nc, numBlocks));
}

// ThrMatrixMultEx2 ThreadedMatrixOperations.pas:612-718: strips of height x width, each a
// BlockMatrixMultiplication (MatrixMultFunc :335-353).  Values are those of the single-threaded
// blocked multiplication because every output entry sees the same k-blocking.
void thr_mult_ex2(double* dest, int64_t lwd, const double* mt1, const double* mt2, int64_t w1, int64_t h1,
                  int64_t w2, int64_t h2, int64_t lw1, int64_t lw2, int64_t bs, int32_t op, bool haveMem) {
    const int used = num_cores_for_mult(w1, h1, w2, h2, bs);
    if (used == 1) {
        block_mult(dest, lwd, mt1, mt2, w1, h1, w2, h2, lw1, lw2, bs, op, haveMem);
        return;
    }
    int64_t cpud2 = used / 2, thrWidth = w2, thrHeight, heightCores;
    if (cpud2 > 1) {
        heightCores = cpud2;
        cpud2 = used / heightCores;
        thrWidth = w2 / cpud2 + ((w2 % cpud2) ? 1 : 0);
        thrWidth += thrWidth & 1;
        thrHeight = h1 / heightCores + ((h1 % heightCores) ? 1 : 0);
    } else {
        cpud2 = 1;
        thrHeight = h1 / used + ((h1 % used) ? 1 : 0);
        thrHeight += thrHeight & 1;
        heightCores = used;
    }
    std::vector<std::function<void()>> tasks;
    for (int64_t j = 0; j < cpud2; ++j) {
        for (int64_t i = 0; i < heightCores; ++i) {
            int64_t hh = (h1 > (i + 1) * thrHeight) ? thrHeight : h1 - i * thrHeight;
            int64_t ww = (w2 > (j + 1) * thrWidth) ? thrWidth : w2 - j * thrWidth;
            if (hh <= 0 || ww <= 0) break;
            double* d = rowp(dest, i * thrHeight, lwd) + j * thrWidth;
            const double* a = rowp(mt1, i * thrHeight, lw1);
            const double* b = mt2 + j * thrWidth;
            const bool useCache = (op == 0 && !haveMem);
            tasks.push_back([=] {
                block_mult(d, lwd, a, b, w1, hh, ww, h2, lw1, lw2, useCache ? 128 : bs, op, haveMem);
            });
        }
    }
    pool()->run(tasks);
}

// ThrBlockMatrixMultiplication BlockedMult.pas:1834-2027 distributes the output blocks of one
// BlockMatrixMultiplication over the pool; restated here as block-column ranges.
void thr_block_mult(double* dest, int64_t lwd, const double* mt1, const double* mt2, int64_t w1, int64_t h1,
                    int64_t w2, int64_t h2, int64_t lw1, int64_t lw2, int64_t bs, int32_t op) {
    const int64_t nbx = w2 / bs + ((w2 % bs) ? 1 : 0);
    const int nc = pool()->size();
    std::vector<std::function<void()>> tasks;
    const int64_t per = (nbx + nc - 1) / nc;
    for (int64_t b0 = 0; b0 < nbx; b0 += per) {
        const int64_t b1 = std::min(nbx, b0 + per);
        tasks.push_back([=] { block_mult_rows(dest, lwd, mt1, mt2, w1, h1, w2, h2, lw1, lw2, bs, op, b0, b1); });
    }
    pool()->run(tasks);
}

// ThrMatrixMultEx ThreadedMatrixOperations.pas:720-729 with UseInnerBlockMult BlockedMult.pas:1646-1650
void thr_mult_ex(double* dest, int64_t lwd, const double* mt1, const double* mt2, int64_t w1, int64_t h1,
                 int64_t w2, int64_t h2, int64_t lw1, int64_t lw2, int64_t bs, int32_t op, bool haveMem) {
    if (w1 < 1024 && h1 < 1024 && w1 > 512 && h1 > 512)
        thr_block_mult(dest, lwd, mt1, mt2, w1, h1, w2, h2, lw1, lw2, bs, op);
    else
        thr_mult_ex2(dest, lwd, mt1, mt2, w1, h1, w2, h2, lw1, lw2, bs, op, haveMem);
}

// ------------------------------------------------------------------------------------
// LU (LinAlgLU.pas)
// ------------------------------------------------------------------------------------
const int64_t kBlkMultSize = 48;  // cBlkMultSize :171

// LUSwap :120-136
void lu_swap(double* A, int64_t lw, int64_t width, int64_t k1, int64_t k2, const int32_t* indx) {
    for (int64_t i = k1; i <= k2; ++i)
        if (indx[i] != i) row_swap(rowp(A, i, lw), rowp(A, indx[i], lw), width);
}

// LUBacksup :138-169: B(height x width) <- L^{-1} B with L unit lower, read from A below the diagonal.
void lu_backsup(const double* A, int64_t width, int64_t height, double* B, int64_t lw) {
    for (int64_t k = 0; k < height; ++k) {
        const double* pB = rowp(B, k, lw);
        for (int64_t i = k + 1; i < height; ++i) {
            const double l = rowp(A, i, lw)[k];
            double* d = rowp(B, i, lw);
            for (int64_t j = 0; j < width; ++j) d[j] = d[j] - pB[j] * l;
        }
    }
}

// ThrMatrixUSubst :627-672: column strips of LUBacksup
void thr_usubst(const double* A, int64_t width, int64_t height, double* B, int64_t lw) {
    const int nc = pool()->size();
    const int64_t thrSize = std::max<int64_t>(32, width / nc + ((width % nc) ? 1 : 0));
    std::vector<std::function<void()>> tasks;
    for (int64_t i = 0; i < nc; ++i) {
        int64_t wSize = thrSize;
        if (wSize * (i + 1) >= width) wSize = width - i * thrSize;
        double* b = B + i * thrSize;
        tasks.push_back([=] { lu_backsup(A, wSize, height, b, lw); });
        if (thrSize * (i + 1) >= width) break;
    }
    pool()->run(tasks);
}

struct RecData {
    int64_t lw;
    std::vector<double> mem;  // BlockMultMemSize(48) scratch
    bool threaded;
    double* gap;              // optional pivot-gap tracker
};

// InternalRecursiveMatrixLUDecompInPlace :181-281 (threaded twin :674-786 when d.threaded)
int32_t rec_lu(double* A, int64_t width, int64_t height, int32_t* indx, RecData& d) {
    const int64_t mn = std::min(width, height);
    const int64_t lw = d.lw;
    if (mn > 1) {
        const int64_t nleft = mn / 2, nright = width - nleft;
        int32_t r = rec_lu(A, nleft, height, indx, d);
        if (r != 0) return r;
        double* pA = A + nleft;
        lu_swap(pA, lw, nright, 0, nleft - 1, indx);
        if (nright > 1) {
            if (d.threaded && nright > 64) thr_usubst(A, nright, nleft, pA, lw);
            else lu_backsup(A, nright, nleft, pA, lw);
        }
        double* a12 = A + nleft;
        double* pB = rowp(A, nleft, lw) + nleft;
        double* a21 = rowp(A, nleft, lw);
        if (nright > kBlkMultSize || height - nleft > kBlkMultSize) {
            if (d.threaded)
                thr_mult_ex(pB, lw, a21, a12, nleft, height - nleft, nright, nleft, lw, lw, kBlkMultSize, 2, true);
            else
                block_mult(pB, lw, a21, a12, nleft, height - nleft, nright, nleft, lw, lw, kBlkMultSize, 2, true);
        } else {
            const int64_t mlw = (nright + (nright & 1)) * 8;
            matrix_mult(d.mem.data(), mlw, a21, a12, nleft, height - nleft, nright, nleft, lw, lw);
            mtx_sub(pB, lw, pB, d.mem.data(), nright, height - nleft, lw, mlw);
        }
        r = rec_lu(pB, nright, height - nleft, indx + nleft, d);
        if (r != 0) return r;
        for (int64_t i = nleft; i < width; ++i) indx[i] += (int32_t)nleft;
        lu_swap(A, lw, nleft, nleft, mn - 1, indx);
        return 0;
    }
    // leaf: one column
    double maxVal = 0.0, absMaxVal = 0.0, second = 0.0;
    int64_t idx = -1;
    for (int64_t i = 0; i < height; ++i) {
        const double v = rowp(A, i, lw)[0];
        if (std::fabs(v) > absMaxVal) {
            second = absMaxVal;
            idx = i;
            maxVal = v;
            absMaxVal = std::fabs(maxVal);
        } else if (std::fabs(v) > second) {
            second = std::fabs(v);
        }
    }
    if (d.gap && height > 1 && absMaxVal > 0.0) *d.gap = std::min(*d.gap, (absMaxVal - second) / absMaxVal);
    indx[0] = (int32_t)idx;
    if (std::fabs(maxVal) > 10.0 / DBL_MAX) {
        // MatrixScaleAndAdd(A, LineWidth, 1, Height, 0, 1/maxVal): x*Scale + Offset
        const double scale = 1.0 / maxVal;
        for (int64_t i = 0; i < height; ++i) {
            double* p = rowp(A, i, lw);
            p[0] = (p[0] * scale) + 0.0;
        }
        rowp(A, idx, lw)[0] = A[0];
        A[0] = maxVal;
        return 0;
    }
    return 1;
}

int32_t lu_inplace(double* A, int64_t lw, int64_t width, int32_t* indx, bool threaded, double* gap) {
    std::memset(indx, 0, width * sizeof(int32_t));
    RecData d;
    d.lw = lw;
    d.mem.assign((size_t)(4 * kBlkMultSize * kBlkMultSize), 0.0);
    d.threaded = threaded;
    d.gap = gap;
    return rec_lu(A, width, width, indx, d);
}

// MatrixLUBackSubst :315-385
void lu_backsubst(const double* LU, int64_t lwLU, int64_t width, const int32_t* indx, double* B, int64_t lwB) {
    int64_t ii = -1;
    for (int64_t i = 0; i < width; ++i) {
        const int64_t ip = indx[i];
        double* pB = rowp(B, ip, lwB);
        double sum = *pB;
        *pB = *rowp(B, i, lwB);
        if (ii >= 0) {
            const double* l = rowp(LU, i, lwLU);
            for (int64_t j = ii; j <= i - 1; ++j) sum = sum - l[j] * *rowp(B, j, lwB);
        } else if (sum != 0.0) {
            ii = i;
        }
        *rowp(B, i, lwB) = sum;
    }
    for (int64_t i = width - 1; i >= 0; --i) {
        double sum = *rowp(B, i, lwB);
        const double* u = rowp(LU, i, lwLU);
        for (int64_t j = i + 1; j < width; ++j) sum = sum - u[j] * *rowp(B, j, lwB);
        *rowp(B, i, lwB) = sum / u[i];
    }
}

// refinement loop of MatrixLinEQSolve :542-586 (and ThrMatrixLinEQSolve :1076-1120)
void refine(const double* A, int64_t lwA, int64_t width, const double* B, int64_t lwB, double* X, int64_t lwX,
            int64_t width2, int64_t numRef, const double* LU, int64_t lwLU, const int32_t* indx, bool rowQuirk) {
    std::vector<double> row((size_t)width);
    for (int64_t k = 0; k < width2; ++k) {
        for (int64_t rc = 0; rc < numRef; ++rc) {
            for (int64_t i = 0; i < width; ++i) {
                const double* a = rowp(A, i, lwA);
                double sdp = -*rowp(B, i, lwB);
                for (int64_t j = 0; j < width; ++j) {
                    const double xv = rowQuirk ? X[j] : *rowp(X, j, lwX);
                    sdp = sdp + xv * a[j];
                }
                row[i] = sdp;
            }
            lu_backsubst(LU, lwLU, width, indx, row.data(), sizeof(double));
            for (int64_t i = 0; i < width; ++i) {
                double* px = rowp(X, i, lwX);
                *px = *px - row[i];
            }
        }
        ++B;
        ++X;
    }
}

double g_dummy_gap = 1.0;

}  // namespace

// ======================================================================================
// exported API
// ======================================================================================
extern "C" void orc_generic_mult(double* dest, int64_t lwd, const double* mt1, const double* mt2, int64_t w1,
                                 int64_t h1, int64_t w2, int64_t h2, int64_t lw1, int64_t lw2) {
    generic_mult(dest, lwd, mt1, mt2, w1, h1, w2, h2, lw1, lw2);
}

extern "C" void orc_matrix_mult(double* dest, int64_t lwd, const double* mt1, const double* mt2, int64_t w1,
                                int64_t h1, int64_t w2, int64_t h2, int64_t lw1, int64_t lw2) {
    matrix_mult(dest, lwd, mt1, mt2, w1, h1, w2, h2, lw1, lw2);
}

extern "C" void orc_block_mult(double* dest, int64_t lwd, const double* mt1, const double* mt2, int64_t w1,
                               int64_t h1, int64_t w2, int64_t h2, int64_t lw1, int64_t lw2, int64_t blockSize,
                               int32_t op) {
    block_mult(dest, lwd, mt1, mt2, w1, h1, w2, h2, lw1, lw2, blockSize, op, false);
}

extern "C" void orc_block_mult_t1(double* dest, int64_t lwd, const double* mt1, const double* mt2, int64_t w1,
                                  int64_t h1, int64_t w2, int64_t h2, int64_t lw1, int64_t lw2, int64_t bs,
                                  int32_t op) {
    // BlockMatrixMultiplicationT1 BlockedMult.pas:477-593: dest(w1 x w2) = mt1(h1 x w1)^T * mt2(h2 x w2)
    if (w1 == 0 || w2 == 0 || h1 == 0 || h2 == 0) return;
    if (bs > w1) bs = next2pwr(h1, bs);
    const bool h1Fit = (h1 % bs) == 0, w2Fit = (w2 % bs) == 0, w1Fit = (w1 % bs) == 0;
    const int64_t nw1 = w1 / bs + (w1Fit ? 0 : 1) - 1;
    const int64_t nw = w2 / bs + (w2Fit ? 0 : 1) - 1;
    const int64_t gamma = h1 / bs + (h1Fit ? 0 : 1) - 1;
    std::vector<double> act((size_t)(bs * bs)), mult((size_t)(bs * bs)), t1((size_t)(bs * bs)), t2((size_t)(bs * bs));
    const int64_t bl = bs * 8;
    for (int64_t by = 0; by <= nw1; ++by) {
        const int64_t bw1 = (by == nw1 && !w1Fit) ? w1 % bs : bs;
        for (int64_t bx = 0; bx <= nw; ++bx) {
            const int64_t bw = (bx == nw && !w2Fit) ? w2 % bs : bs;
            std::fill(act.begin(), act.end(), 0.0);
            const double* pa = mt1 + by * bs;
            const double* pb = mt2 + bx * bs;
            for (int64_t idx = 0; idx <= gamma; ++idx) {
                const int64_t gh = (idx == gamma && !h1Fit) ? h1 % bs : bs;
                mtx_transpose(t1.data(), bl, pa, lw1, bw1, gh);
                if (bw > 3 && bw1 > 3) {
                    mtx_transpose(t2.data(), bl, pb, lw2, bw, gh);
                    matrix_multT2(mult.data(), bl, t1.data(), t2.data(), gh, bw1, bw, bl, bl);
                } else {
                    generic_mult(mult.data(), bl, t1.data(), pb, gh, bw1, bw, gh, bl, lw2);
                }
                mtx_add(act.data(), bl, act.data(), mult.data(), bw, bw1, bl, bl);
                pa = rowp(pa, gh, lw1);
                pb = rowp(pb, gh, lw2);
            }
            double* pDest = rowp(dest, by * bs, lwd) + bx * bs;
            if (op == 0) mtx_copy(pDest, lwd, act.data(), bl, bw, bw1);
            else if (op == 1) mtx_add(pDest, lwd, pDest, act.data(), bw, bw1, lwd, bl);
            else mtx_sub(pDest, lwd, pDest, act.data(), bw, bw1, lwd, bl);
        }
    }
}

extern "C" void orc_block_mult_t2(double* dest, int64_t lwd, const double* mt1, const double* mt2, int64_t w1,
                                  int64_t h1, int64_t w2, int64_t h2, int64_t lw1, int64_t lw2, int64_t bs,
                                  int32_t op) {
    // BlockMatrixMultiplicationT2 BlockedMult.pas:596-724: dest(h1 x h2) = mt1(h1 x w1) * mt2(h2 x w2)^T
    if (w1 == 0 || w2 == 0 || h1 == 0 || h2 == 0) return;
    if (op == 0 && w1 <= bs) {  // shortcut :628-632
        matrix_multT2(dest, lwd, mt1, mt2, w1, h1, h2, lw1, lw2);
        return;
    }
    if (bs > w1) bs = next2pwr(w1, bs);
    const bool h1Fit = (h1 % bs) == 0, h2Fit = (h2 % bs) == 0, w1Fit = (w1 % bs) == 0;
    const int64_t nh = h1 / bs + (h1Fit ? 0 : 1) - 1;
    const int64_t nh1 = h2 / bs + (h2Fit ? 0 : 1) - 1;
    const int64_t gamma = w1 / bs + (w1Fit ? 0 : 1) - 1;
    std::vector<double> act((size_t)(bs * bs)), mult((size_t)(bs * bs));
    const int64_t bl = bs * 8;
    for (int64_t by = 0; by <= nh; ++by) {
        const int64_t bh = (by == nh && !h1Fit) ? h1 % bs : bs;
        for (int64_t bx = 0; bx <= nh1; ++bx) {
            const int64_t bh1 = (bx == nh1 && !h2Fit) ? h2 % bs : bs;
            std::fill(act.begin(), act.end(), 0.0);
            const double* pa = rowp(mt1, by * bs, lw1);
            const double* pb = rowp(mt2, bx * bs, lw2);
            for (int64_t idx = 0; idx <= gamma; ++idx) {
                const int64_t gw = (idx == gamma && !w1Fit) ? w1 % bs : bs;
                if (bh1 > 3 && bh > 3)
                    matrix_multT2(mult.data(), bl, pa, pb, gw, bh, bh1, lw1, lw2);
                else
                    generic_mult_transp(mult.data(), bl, pa, pb, gw, bh, gw, bh1, lw1, lw2);
                mtx_add(act.data(), bl, act.data(), mult.data(), bh1, bh, bl, bl);
                pa += gw;
                pb += gw;
            }
            double* pDest = rowp(dest, by * bs, lwd) + bx * bs;
            if (op == 0) mtx_copy(pDest, lwd, act.data(), bl, bh1, bh);
            else if (op == 1) mtx_add(pDest, lwd, pDest, act.data(), bh1, bh, lwd, bl);
            else mtx_sub(pDest, lwd, pDest, act.data(), bh1, bh, lwd, bl);
        }
    }
}

extern "C" int32_t orc_lu_decomp_inplace(double* A, int64_t lwA, int64_t width, int32_t* indx) {
    return lu_inplace(A, lwA, width, indx, false, nullptr);
}

extern "C" int32_t orc_lu_decomp(const double* A, int64_t lwA, double* LU, int64_t lwLU, int64_t width,
                                 int32_t* indx) {
    mtx_copy(LU, lwLU, A, lwA, width, width);
    return lu_inplace(LU, lwLU, width, indx, false, nullptr);
}

extern "C" void orc_lu_backsubst(const double* LU, int64_t lwLU, int64_t width, const int32_t* indx, double* B,
                                 int64_t lwB) {
    lu_backsubst(LU, lwLU, width, indx, B, lwB);
}

extern "C" int32_t orc_inverse_inplace(double* A, int64_t lwA, int64_t width) {
    // MatrixInverseInPlace :388-431
    const int64_t w = width + (width & 1);
    std::vector<double> Y((size_t)(w * w));
    std::vector<int32_t> indx((size_t)width);
    std::vector<double> col((size_t)width);
    mtx_copy(Y.data(), w * 8, A, lwA, width, width);
    if (lu_inplace(Y.data(), w * 8, width, indx.data(), false, nullptr) == 1) return 1;
    for (int64_t j = 0; j < width; ++j) {
        std::fill(col.begin(), col.end(), 0.0);
        col[j] = 1.0;
        lu_backsubst(Y.data(), w * 8, width, indx.data(), col.data(), 8);
        for (int64_t i = 0; i < width; ++i) rowp(A, i, lwA)[j] = col[i];
    }
    return 0;
}

static double determinant_impl(const double* A, int64_t lwA, int64_t width, bool threaded) {
    // MatrixDeterminant :433-479 (w rounded up to even) / ThrMatrixDeterminant (w rounded to 4)
    int64_t w = width;
    if (threaded) { if (w & 3) w += 4 - (width & 3); }
    else w = width + (width & 1);
    std::vector<double> LU((size_t)(w * width));
    std::vector<int32_t> indx((size_t)width);
    mtx_copy(LU.data(), w * 8, A, lwA, width, width);
    if (lu_inplace(LU.data(), w * 8, width, indx.data(), threaded, nullptr) == 1) return 0.0;
    double res = 1.0;
    for (int64_t i = 0; i < width; ++i)
        if (indx[i] != i) res = -res;
    for (int64_t i = 0; i < width; ++i) res = res * LU[(size_t)(i * w + i)];
    return res;
}

extern "C" double orc_determinant(const double* A, int64_t lwA, int64_t width) {
    return determinant_impl(A, lwA, width, false);
}

extern "C" int32_t orc_lineq_solve(const double* A, int64_t lwA, int64_t width, const double* B, int64_t lwB,
                                   double* X, int64_t lwX, int64_t width2, int64_t numRef, int32_t rowQuirk) {
    // MatrixLinEQSolve :481-592: contiguous LU with stride width*8 (:510)
    std::vector<double> LU((size_t)(width * width));
    std::vector<int32_t> indx((size_t)width);
    mtx_copy(LU.data(), width * 8, A, lwA, width, width);
    if (lu_inplace(LU.data(), width * 8, width, indx.data(), false, nullptr) == 1) return 1;
    for (int64_t i = 0; i < width2; ++i) {
        for (int64_t j = 0; j < width; ++j) rowp(X, j, lwX)[i] = rowp(B, j, lwB)[i];
        lu_backsubst(LU.data(), width * 8, width, indx.data(), X + i, lwX);
    }
    if (numRef > 0)
        refine(A, lwA, width, B, lwB, X, lwX, width2, numRef, LU.data(), width * 8, indx.data(), rowQuirk != 0);
    return 0;
}

extern "C" void orc_set_num_threads(int32_t n) {
    g_threads = n;
    if (g_threads <= 0) g_threads = std::max(1L, sysconf(_SC_NPROCESSORS_ONLN));
    g_threads = std::min(g_threads, 64);
    pool()->resize(g_threads);
}
extern "C" int32_t orc_get_num_threads(void) { return pool()->size(); }

extern "C" void orc_thr_matrix_mult(double* dest, int64_t lwd, const double* mt1, const double* mt2, int64_t w1,
                                    int64_t h1, int64_t w2, int64_t h2, int64_t lw1, int64_t lw2, int64_t blockSize,
                                    int32_t op) {
    thr_mult_ex(dest, lwd, mt1, mt2, w1, h1, w2, h2, lw1, lw2, blockSize, op, false);
}

extern "C" int32_t orc_thr_lu_decomp(double* A, int64_t lwA, int64_t width, int32_t* indx) {
    return lu_inplace(A, lwA, width, indx, true, nullptr);
}

extern "C" int32_t orc_thr_lineq_solve(const double* A, int64_t lwA, int64_t width, const double* B, int64_t lwB,
                                       double* X, int64_t lwX, int64_t width2, int64_t numRef) {
    // ThrMatrixLinEQSolve :986-1128: LU rows padded to a multiple of 4 doubles
    int64_t w = width;
    if (w & 3) w += 4 - (width & 3);
    const int64_t lwLU = w * 8;
    std::vector<double> LU((size_t)(w * width));
    std::vector<int32_t> indx((size_t)width);
    mtx_copy(LU.data(), lwLU, A, lwA, width, width);
    if (lu_inplace(LU.data(), lwLU, width, indx.data(), true, nullptr) == 1) return 1;
    mtx_copy(X, lwX, B, lwB, width2, width);
    const int nc = pool()->size();
    const int64_t thrSize = std::max<int64_t>(1, width2 / nc + ((width2 % nc) ? 1 : 0));
    const int64_t nt = std::min<int64_t>(thrSize, nc);
    std::vector<std::function<void()>> tasks;
    for (int64_t i = 0; i < nt; ++i) {
        int64_t wSize = thrSize;
        if (i == nt - 1) wSize = width2 - i * thrSize;
        const int64_t off = i * thrSize;
        tasks.push_back([=, &LU, &indx] {
            for (int64_t j = 0; j < wSize; ++j) lu_backsubst(LU.data(), lwLU, width, indx.data(), X + off + j, lwX);
        });
    }
    pool()->run(tasks);
    if (numRef > 0) refine(A, lwA, width, B, lwB, X, lwX, width2, numRef, LU.data(), lwLU, indx.data(), true);
    return 0;
}

extern "C" int32_t orc_thr_inverse(double* A, int64_t lwA, int64_t width) {
    // ThrMatrixInverse :853-929
    int64_t w = width;
    if (w & 3) w += 4 - (width & 3);
    const int64_t lwY = w * 8;
    std::vector<double> Y((size_t)(w * width));
    std::vector<int32_t> indx((size_t)width);
    mtx_copy(Y.data(), lwY, A, lwA, width, width);
    if (lu_inplace(Y.data(), lwY, width, indx.data(), true, nullptr) == 1) return 1;
    const int nc = pool()->size();
    const int64_t thrSize = std::max<int64_t>(32, width / nc + ((width % nc) ? 1 : 0));
    std::vector<std::function<void()>> tasks;
    for (int64_t i = 0; i < nc; ++i) {
        int64_t wSize = thrSize;
        if (wSize * (i + 1) > width) wSize = width - i * thrSize;
        const int64_t off = i * thrSize;
        const int64_t cnt = std::min(wSize, width);
        tasks.push_back([=, &Y, &indx] {
            std::vector<double> col((size_t)width);
            for (int64_t j = 0; j < cnt; ++j) {
                std::fill(col.begin(), col.end(), 0.0);
                col[j + off] = 1.0;
                lu_backsubst(Y.data(), lwY, width, indx.data(), col.data(), 8);
                for (int64_t r = 0; r < width; ++r) rowp(A, r, lwA)[off + j] = col[r];
            }
        });
        if ((i + 1) * thrSize >= width) break;
    }
    pool()->run(tasks);
    return 0;
}

extern "C" double orc_thr_determinant(const double* A, int64_t lwA, int64_t width) {
    return determinant_impl(A, lwA, width, true);
}

extern "C" double orc_lu_min_pivot_gap(const double* A, int64_t lwA, int64_t width) {
    std::vector<double> LU((size_t)(width * width));
    std::vector<int32_t> indx((size_t)width);
    mtx_copy(LU.data(), width * 8, A, lwA, width, width);
    double gap = 1.0;
    lu_inplace(LU.data(), width * 8, width, indx.data(), false, &gap);
    (void)g_dummy_gap;
    return gap;
}

// ---------------- compensated arithmetic (Ogita, Rump, Oishi 2005, "Accurate sum and dot product") --------------
namespace {
inline void two_sum(double a, double b, double& s, double& e) {
    s = a + b;
    double z = s - a;
    e = (a - (s - z)) + (b - z);
}
inline void two_prod(double a, double b, double& p, double& e) {
    p = a * b;
    e = std::fma(a, b, -p);
}
}  // namespace

extern "C" void orc_residual_dot2(const double* A, int64_t lwA, int64_t n, const double* X, int64_t lwX,
                                  const double* B, int64_t lwB, int64_t nrhs, double* R, int64_t lwR) {
    // rows are independent: split them over the pool (each entry is one sequential Dot2 sum)
    std::vector<std::function<void()>> tasks;
    const int nt = pool()->size();
    const int64_t per = std::max<int64_t>(1, (n + nt - 1) / nt);
    for (int64_t i0 = 0; i0 < n; i0 += per) {
        const int64_t i1 = std::min(n, i0 + per);
        tasks.push_back([=] {
            for (int64_t i = i0; i < i1; ++i) {
                const double* a = rowp(A, i, lwA);
                for (int64_t c = 0; c < nrhs; ++c) {
                    double s = rowp(B, i, lwB)[c], comp = 0.0;
                    for (int64_t j = 0; j < n; ++j) {
                        double p, ep, t, et;
                        two_prod(-a[j], rowp(X, j, lwX)[c], p, ep);
                        two_sum(s, p, t, et);
                        s = t;
                        comp = comp + (et + ep);
                    }
                    rowp(R, i, lwR)[c] = s + comp;
                }
            }
        });
    }
    pool()->run(tasks);
}

extern "C" double orc_backward_error(const double* A, int64_t lwA, int64_t n, const double* X, int64_t lwX,
                                     const double* B, int64_t lwB, int64_t nrhs) {
    std::vector<double> R((size_t)(n * nrhs));
    orc_residual_dot2(A, lwA, n, X, lwX, B, lwB, nrhs, R.data(), nrhs * 8);
    double normA = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        double s = 0.0;
        const double* a = rowp(A, i, lwA);
        for (int64_t j = 0; j < n; ++j) s += std::fabs(a[j]);
        normA = std::max(normA, s);
    }
    double eta = 0.0;
    for (int64_t c = 0; c < nrhs; ++c) {
        double rn = 0.0, xn = 0.0, bn = 0.0;
        for (int64_t i = 0; i < n; ++i) {
            rn = std::max(rn, std::fabs(R[(size_t)(i * nrhs + c)]));
            xn = std::max(xn, std::fabs(rowp(X, i, lwX)[c]));
            bn = std::max(bn, std::fabs(rowp(B, i, lwB)[c]));
        }
        eta = std::max(eta, rn / (normA * xn + bn));
    }
    return eta;
}

// ---------------- complex LU (LinAlgLU.pas:1147-1603) ---------------------------------------------------------
// TComplex = record real, imag : double (16 bytes); the arithmetic helpers of CplxSimpleMatrixOperations.pas
// are restated with their evaluation order (the oracle is compiled without FP contraction).
namespace {

struct Cx {
    double re, im;
};
inline Cx* crow(void* A, int64_t r, int64_t lw) { return reinterpret_cast<Cx*>(static_cast<char*>(A) + r * lw); }
inline const Cx* crow(const void* A, int64_t r, int64_t lw) {
    return reinterpret_cast<const Cx*>(static_cast<const char*>(A) + r * lw);
}
inline double cabs1(Cx v) { return std::fabs(v.re) + std::fabs(v.im); }                       // :208-211
inline void cinc_mul(Cx& x1, Cx x2, Cx x3) {                                                   // CIncMul
    x1.re = x1.re + x2.re * x3.re - x2.im * x3.im;
    x1.im = x1.im + x2.re * x3.im + x2.im * x3.re;
}
inline Cx cadd_mul(Cx x1, Cx x2, Cx x3) {                                                      // CAddMul
    return Cx{x1.re + x2.re * x3.re - x2.im * x3.im, x1.im + x2.re * x3.im + x2.im * x3.re};
}
inline Cx csub_mul(Cx x1, Cx x2, Cx x3) {                                                      // CSubMul
    return Cx{x1.re - x2.re * x3.re + x2.im * x3.im, x1.im - x2.re * x3.im - x2.im * x3.re};
}
inline Cx cmul(Cx a, Cx b) { return Cx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }  // CMul
inline Cx cdiv(Cx x1, Cx x2) {                                                                 // CDiv (Smith)
    if (std::fabs(x2.re) >= std::fabs(x2.im)) {
        const double r = x2.im / x2.re, den = x2.re + x2.im * r;
        return Cx{(x1.re + r * x1.im) / den, (x1.im - r * x1.re) / den};
    }
    const double r = x2.re / x2.im, den = x2.im + x2.re * r;
    return Cx{(x1.re * r + x1.im) / den, (x1.im * r - x1.re) / den};
}
inline Cx cinv(Cx x1) {                                                                        // CInv
    if (std::fabs(x1.re) >= std::fabs(x1.im)) {
        const double r = x1.im / x1.re, den = x1.re + x1.im * r;
        return Cx{1.0 / den, -r / den};
    }
    const double r = x1.re / x1.im, den = x1.im + r * x1.re;
    return Cx{r / den, -1.0 / den};
}

// CplxGenericMtxMult CplxSimpleMatrixOperations.pas:983-1013: dest = mt1 mt2, sums from (0, 0) in order
void cplx_mult(void* dest, int64_t lwd, const void* mt1, const void* mt2, int64_t w1, int64_t h1, int64_t w2,
               int64_t lw1, int64_t lw2) {
    for (int64_t y = 0; y < h1; ++y)
        for (int64_t x = 0; x < w2; ++x) {
            Cx s{0.0, 0.0};
            for (int64_t k = 0; k < w1; ++k) cinc_mul(s, crow(mt1, y, lw1)[k], crow(mt2, k, lw2)[x]);
            crow(dest, y, lwd)[x] = s;
        }
}

// CplxGenericBlockMatrixMultiplication BlockedMult.pas:837-920 with op doSub: dest -= mt1 mt2 through
// blockSize blocks, each block's products summed over the k-blocks into actBlk, then subtracted
void cplx_block_mult_sub(void* dest, int64_t lwd, const void* mt1, const void* mt2, int64_t w1, int64_t h1,
                         int64_t w2, int64_t lw1, int64_t lw2, int64_t bs) {
    if (w1 == 0 || w2 == 0 || h1 == 0) return;
    const bool h1Fit = (h1 % bs) == 0, w2Fit = (w2 % bs) == 0, w1Fit = (w1 % bs) == 0;
    const int64_t h = h1 / bs + (h1Fit ? 0 : 1) - 1, w = w2 / bs + (w2Fit ? 0 : 1) - 1;
    const int64_t gamma = w1 / bs + (w1Fit ? 0 : 1) - 1;
    std::vector<Cx> act((size_t)(bs * bs)), mult((size_t)(bs * bs));
    const int64_t bl = bs * 16;
    for (int64_t by = 0; by <= h; ++by) {
        const int64_t bh = (by == h && !h1Fit) ? h1 % bs : bs;
        for (int64_t bx = 0; bx <= w; ++bx) {
            const int64_t bw = (bx == w && !w2Fit) ? w2 % bs : bs;
            std::fill(act.begin(), act.end(), Cx{0.0, 0.0});
            for (int64_t idx = 0; idx <= gamma; ++idx) {
                const int64_t gw = (idx == gamma && !w1Fit) ? w1 % bs : bs;
                const Cx* pa = crow(mt1, by * bs, lw1) + idx * bs;
                const Cx* pb = crow(mt2, idx * bs, lw2) + bx * bs;
                cplx_mult(mult.data(), bl, pa, pb, gw, bh, bw, lw1, lw2);
                for (int64_t y = 0; y < bh; ++y)
                    for (int64_t x = 0; x < bw; ++x) {
                        Cx& a = act[(size_t)(y * bs + x)];
                        const Cx m = mult[(size_t)(y * bs + x)];
                        a = Cx{a.re + m.re, a.im + m.im};
                    }
            }
            for (int64_t y = 0; y < bh; ++y)
                for (int64_t x = 0; x < bw; ++x) {
                    Cx& d = crow(dest, by * bs + y, lwd)[bx * bs + x];
                    const Cx a = act[(size_t)(y * bs + x)];
                    d = Cx{d.re - a.re, d.im - a.im};
                }
        }
    }
}

void cplx_lu_swap(void* A, int64_t lw, int64_t width, int64_t k1, int64_t k2, const int32_t* indx) {  // :1183-1200
    for (int64_t i = k1; i <= k2; ++i)
        if (indx[i] != i)
            for (int64_t x = 0; x < width; ++x) std::swap(crow(A, i, lw)[x], crow(A, indx[i], lw)[x]);
}

void cplx_lu_backsup(const void* A, int64_t width, int64_t height, void* B, int64_t lw) {  // :1147-1181
    for (int64_t k = 0; k < height; ++k)
        for (int64_t i = k + 1; i < height; ++i) {
            const Cx aik = crow(A, i, lw)[k];
            for (int64_t j = 0; j < width; ++j)
                crow(B, i, lw)[j] = csub_mul(crow(B, i, lw)[j], crow(B, k, lw)[j], aik);
        }
}

// InternalRecursiveCplxMatrixLUDecompInPlace :1202-1306 (cBlkMultSize = 48)
int32_t cplx_rec_lu(void* A, int64_t width, int64_t height, int32_t* indx, int64_t lw) {
    const int64_t mn = std::min(width, height);
    if (mn > 1) {
        const int64_t nleft = mn / 2, nright = width - nleft;
        int32_t r = cplx_rec_lu(A, nleft, height, indx, lw);
        if (r != 0) return r;
        Cx* pA = crow(A, 0, lw) + nleft;
        cplx_lu_swap(pA, lw, nright, 0, nleft - 1, indx);
        if (nright > 1) cplx_lu_backsup(A, nright, nleft, pA, lw);
        Cx* pB = crow(A, nleft, lw) + nleft;
        const Cx* a21 = crow(A, nleft, lw);
        if (nright > 48 || height - nleft > 48) {
            cplx_block_mult_sub(pB, lw, a21, pA, nleft, height - nleft, nright, lw, lw, 48);
        } else {
            const int64_t lwb = (nright + (nright & 1)) * 16;
            std::vector<Cx> mem((size_t)((nright + 1) * (height - nleft + 1)));
            cplx_mult(mem.data(), lwb, a21, pA, nleft, height - nleft, nright, lw, lw);
            for (int64_t y = 0; y < height - nleft; ++y)
                for (int64_t x = 0; x < nright; ++x) {
                    Cx& d = crow(pB, y, lw)[x];
                    const Cx m = crow(mem.data(), y, lwb)[x];
                    d = Cx{d.re - m.re, d.im - m.im};
                }
        }
        r = cplx_rec_lu(pB, nright, height - nleft, indx + nleft, lw);
        if (r != 0) return r;
        for (int64_t i = nleft; i < width; ++i) indx[i] += (int32_t)nleft;
        cplx_lu_swap(A, lw, nleft, nleft, mn - 1, indx);
        return 0;
    }
    Cx maxVal{0.0, 0.0};
    double absMax = 0.0;
    int64_t idx = -1;
    for (int64_t i = 0; i < height; ++i) {
        const double av = cabs1(crow(A, i, lw)[0]);
        if (av > absMax) {
            idx = i;
            maxVal = crow(A, i, lw)[0];
            absMax = av;
        }
    }
    indx[0] = (int32_t)idx;
    if (absMax > 10.0 / DBL_MAX) {
        const Cx s = cinv(maxVal);  // CplxGenericMtxScaleAndAdd(A, LW, 1, Height, 0, CInv(maxVal)): x := 0 + x*s
        for (int64_t i = 0; i < height; ++i) crow(A, i, lw)[0] = cadd_mul(Cx{0.0, 0.0}, crow(A, i, lw)[0], s);
        crow(A, idx, lw)[0] = crow(A, 0, lw)[0];
        crow(A, 0, lw)[0] = maxVal;
        return 0;
    }
    return 1;
}

// CplxMatrixLUBackSubst :1322-1391 on one column of B
void cplx_backsubst(const void* LU, int64_t lwLU, int64_t width, const int32_t* indx, void* B, int64_t lwB) {
    int64_t ii = -1;
    for (int64_t i = 0; i < width; ++i) {
        const int64_t ip = indx[i];
        Cx sum = crow(B, ip, lwB)[0];
        crow(B, ip, lwB)[0] = crow(B, i, lwB)[0];
        if (ii >= 0) {
            for (int64_t j = ii; j < i; ++j) sum = csub_mul(sum, crow(LU, i, lwLU)[j], crow(B, j, lwB)[0]);
        } else if (!(std::fabs(sum.re) <= 1e-12 && std::fabs(sum.im) <= 1e-12)) {
            // CCmp(sum, cCplxZero) <> 0: CompareValue with eps 0 takes the RTL's zero resolution, 1e-12
            ii = i;
        }
        crow(B, i, lwB)[0] = sum;
    }
    for (int64_t i = width - 1; i >= 0; --i) {
        Cx sum = crow(B, i, lwB)[0];
        for (int64_t j = 0; j < width - i - 1; ++j)
            sum = csub_mul(sum, crow(LU, i, lwLU)[i + 1 + j], crow(B, i + 1 + j, lwB)[0]);
        crow(B, i, lwB)[0] = cdiv(sum, crow(LU, i, lwLU)[i]);
    }
}

}  // namespace

extern "C" int32_t orc_cplx_lu_decomp_inplace(double* A, int64_t lwA, int64_t width, int32_t* indx) {
    std::fill(indx, indx + width, 0);  // CplxMatrixLUDecompInPlace :1308-1320
    return cplx_rec_lu(A, width, width, indx, lwA);
}

extern "C" void orc_cplx_lu_backsubst(const double* LU, int64_t lwLU, int64_t width, const int32_t* indx, double* B,
                                      int64_t lwB) {
    cplx_backsubst(LU, lwLU, width, indx, B, lwB);
}

extern "C" int32_t orc_cplx_lineq_solve(const double* A, int64_t lwA, int64_t width, const double* B, int64_t lwB,
                                        double* X, int64_t lwX, int64_t nrhs) {
    // CplxMatrixLinEQSolve :1393-1508 without refinement: a contiguous copy of A factored, then one
    // back substitution per column of B
    std::vector<Cx> lu((size_t)(width * width));
    for (int64_t y = 0; y < width; ++y)
        for (int64_t x = 0; x < width; ++x) lu[(size_t)(y * width + x)] = crow(A, y, lwA)[x];
    std::vector<int32_t> indx((size_t)width);
    const int32_t r = orc_cplx_lu_decomp_inplace(reinterpret_cast<double*>(lu.data()), width * 16, width, indx.data());
    if (r != 0) return r;
    std::vector<Cx> col((size_t)width);
    for (int64_t c = 0; c < nrhs; ++c) {
        for (int64_t y = 0; y < width; ++y) col[(size_t)y] = crow(B, y, lwB)[c];
        cplx_backsubst(lu.data(), width * 16, width, indx.data(), col.data(), 16);
        for (int64_t y = 0; y < width; ++y) crow(X, y, lwX)[c] = col[(size_t)y];
    }
    return 0;
}

extern "C" int32_t orc_cplx_inverse_inplace(double* A, int64_t lwA, int64_t width) {
    // CplxMatrixInverseInPlace :1510-1552 (width rounded up to even for the factor's stride)
    const int64_t w = width + (width & 1);
    std::vector<Cx> Y((size_t)(w * w));
    for (int64_t y = 0; y < width; ++y)
        for (int64_t x = 0; x < width; ++x) Y[(size_t)(y * w + x)] = crow(A, y, lwA)[x];
    std::vector<int32_t> indx((size_t)width);
    const int32_t r = orc_cplx_lu_decomp_inplace(reinterpret_cast<double*>(Y.data()), w * 16, width, indx.data());
    if (r != 0) return r;
    std::vector<Cx> col((size_t)width);
    for (int64_t j = 0; j < width; ++j) {
        std::fill(col.begin(), col.end(), Cx{0.0, 0.0});
        col[(size_t)j] = Cx{1.0, 0.0};
        cplx_backsubst(Y.data(), w * 16, width, indx.data(), col.data(), 16);
        for (int64_t i = 0; i < width; ++i) crow(A, i, lwA)[j] = col[(size_t)i];
    }
    return 0;
}

extern "C" void orc_cplx_determinant(const double* A, int64_t lwA, int64_t width, double* det) {
    // CplxMatrixDeterminant :1554-1603: (+-1, 0) times the diagonal of U, in order
    const int64_t w = width + (width & 1);
    std::vector<Cx> lu((size_t)(w * w));
    for (int64_t y = 0; y < width; ++y)
        for (int64_t x = 0; x < width; ++x) lu[(size_t)(y * w + x)] = crow(A, y, lwA)[x];
    std::vector<int32_t> indx((size_t)width);
    if (cplx_rec_lu(lu.data(), width, width, indx.data(), w * 16) != 0) {
        det[0] = det[1] = 0.0;
        return;
    }
    int parity = 1;
    for (int64_t i = 0; i < width; ++i)
        if (indx[(size_t)i] != i) parity = -parity;
    Cx r{(double)parity, 0.0};
    for (int64_t i = 0; i < width; ++i) r = cmul(r, lu[(size_t)(i * w + i)]);
    det[0] = r.re;
    det[1] = r.im;
}

// ---------------- Cholesky (LinAlgCholesky.pas) ------------------------------------------------------------
namespace {

// GenericSymRankKUpd SimpleMatrixOperations.pas:3391-3423: lower triangle of dest (height x height)
// = Beta*dest + Alpha*A A^T, A height x k, the inner sums in ascending l
void sym_rank_k_upd(double* dest, int64_t lwd, const double* A, int64_t lwA, int64_t k, int64_t height, double alpha,
                    double beta) {
    if (k <= 0 || height <= 0) return;
    for (int64_t j = 0; j < height; ++j) {
        double* c = rowp(dest, j, lwd);
        const double* aj = rowp(A, j, lwA);
        for (int64_t i = 0; i <= j; ++i) {
            const double* ai = rowp(A, i, lwA);
            double temp = 0.0;
            for (int64_t l = 0; l < k; ++l) temp = temp + ai[l] * aj[l];
            c[i] = beta * c[i] + alpha * temp;
        }
    }
}

// GenericSolveLoTriMtxTranspNoUnit SimpleMatrixOperations.pas:3463-3510: B (height x width) <- B L^-T,
// column k scaled by the reciprocal 1/L[k][k], then eliminated from the later columns
void solve_lo_tri_transp(const double* A, int64_t lwA, double* B, int64_t lwB, int64_t width, int64_t height) {
    if (width == 0 || height == 0) return;
    for (int64_t k = 0; k < width; ++k) {
        const double temp = 1.0 / rowp(A, k, lwA)[k];
        for (int64_t i = 0; i < height; ++i) rowp(B, i, lwB)[k] = temp * rowp(B, i, lwB)[k];
        for (int64_t j = k + 1; j < width; ++j) {
            const double ajk = rowp(A, j, lwA)[k];
            if (ajk != 0.0)
                for (int64_t i = 0; i < height; ++i)
                    rowp(B, i, lwB)[j] = rowp(B, i, lwB)[j] - ajk * rowp(B, i, lwB)[k];
        }
    }
}

// MatrixCholeskyInPlace2 LinAlgCholesky.pas:205-250: row-oriented unblocked lower Cholesky
int32_t chol_inplace2(double* A, int64_t lwA, int64_t width) {
    for (int64_t i = 0; i < width; ++i) {
        double* ai = rowp(A, i, lwA);
        for (int64_t j = 0; j <= i; ++j) {
            double sum = ai[j];
            const double* aj = rowp(A, j, lwA);
            for (int64_t k = 0; k < j; ++k) sum = sum - ai[k] * aj[k];
            if (i > j)
                ai[j] = sum / aj[j];
            else if (sum > 0)
                ai[i] = std::sqrt(sum);
            else
                return 1;  // crNoPositiveDefinite
        }
    }
    return 0;
}

// InternalBlkCholeskyInPlace LinAlgCholesky.pas:54-103 (left-looking, panels of pnl columns)
int32_t chol_blocked(double* A, int64_t lwA, int64_t width, int64_t pnl) {
    for (int64_t j = 0; j < width; j += pnl) {
        const int64_t jb = std::min(pnl, width - j);
        double* ajj = rowp(A, j, lwA) + j;
        const double* a1 = rowp(A, j, lwA);
        sym_rank_k_upd(ajj, lwA, a1, lwA, j, jb, -1.0, 1.0);
        if (chol_inplace2(ajj, lwA, jb) != 0) return 1;
        if (j + jb < width) {
            double* ajb = rowp(A, j + jb, lwA);
            const double* aj = rowp(A, j, lwA);
            // MatrixMultT2Ex(pAjjb, ..., pAjb, pAj, j, width - j - jb, j, jb, ..., jb, doSub, multMem)
            orc_block_mult_t2(ajb + j, lwA, ajb, aj, j, width - j - jb, j, jb, lwA, lwA, jb, 2);
            solve_lo_tri_transp(ajj, lwA, ajb + j, lwA, jb, width - j - jb);
        }
    }
    return 0;
}

}  // namespace

extern "C" int32_t orc_cholesky_inplace4(double* A, int64_t lwA, int64_t width, int64_t pnl) {
    // MatrixCholeskyInPlace4 LinAlgCholesky.pas:106-123 (pnlSize 0 = CholBlockSize = 32)
    if (pnl == 0) pnl = 32;
    if (width <= pnl) return chol_inplace2(A, lwA, width);
    return chol_blocked(A, lwA, width, pnl);
}

extern "C" int32_t orc_cholesky_inplace2(double* A, int64_t lwA, int64_t width) { return chol_inplace2(A, lwA, width); }

extern "C" int32_t orc_cholesky_nr(double* A, int64_t lwA, int64_t width, double* P, int64_t lwP) {
    // MatrixCholeskyInPlace LinAlgCholesky.pas:270-332: L below the diagonal of A, its diagonal in P
    // (P[i] at byte offset i*lwP); sums run k = i-1 down to 0
    for (int64_t i = 0; i < width; ++i) {
        const double* ai = rowp(A, i, lwA);
        for (int64_t j = i; j < width; ++j) {
            double* aj = rowp(A, j, lwA);
            double sum = ai[j];
            for (int64_t k = i - 1; k >= 0; --k) sum = sum - ai[k] * aj[k];
            if (i == j) {
                if (sum <= 0) return 1;
                rowp(P, i, lwP)[0] = std::sqrt(sum);
            } else {
                aj[i] = sum / rowp(P, i, lwP)[0];
            }
        }
    }
    return 0;
}

extern "C" void orc_cholesky_solve_nr(const double* A, int64_t lwA, int64_t width, const double* P, int64_t lwP,
                                      const double* B, int64_t lwB, double* X, int64_t lwX) {
    // MatrixCholeskySolveLinEq LinAlgCholesky.pas:352-421: L y = b (k descending), L^T x = y (k ascending)
    for (int64_t i = 0; i < width; ++i) {
        double sum = rowp(B, i, lwB)[0];
        const double* ai = rowp(A, i, lwA);
        for (int64_t k = i - 1; k >= 0; --k) sum = sum - ai[k] * rowp(X, k, lwX)[0];
        rowp(X, i, lwX)[0] = sum / rowp(P, i, lwP)[0];
    }
    for (int64_t i = width - 1; i >= 0; --i) {
        double sum = rowp(X, i, lwX)[0];
        for (int64_t k = i + 1; k < width; ++k) sum = sum - rowp(A, k, lwA)[i] * rowp(X, k, lwX)[0];
        rowp(X, i, lwX)[0] = sum / rowp(P, i, lwP)[0];
    }
}

extern "C" void orc_gemm_rows_dot2(const double* A, int64_t lwA, const double* B, int64_t lwB, int64_t /*m*/,
                                   int64_t n, int64_t k, int64_t r0, int64_t nr, double* C, int64_t lwC,
                                   double* absAB, int64_t lwAbs) {
    std::vector<std::function<void()>> tasks;
    const int nc = pool()->size();
    const int64_t per = (nr + nc - 1) / nc;
    for (int64_t t0 = 0; t0 < nr; t0 += per) {
        const int64_t t1 = std::min(nr, t0 + per);
        tasks.push_back([=] {
            for (int64_t ii = t0; ii < t1; ++ii) {
                const double* a = rowp(A, r0 + ii, lwA);
                for (int64_t j = 0; j < n; ++j) {
                    double s = 0.0, comp = 0.0, abs_s = 0.0;
                    for (int64_t q = 0; q < k; ++q) {
                        const double bv = rowp(B, q, lwB)[j];
                        double p, ep, t, et;
                        two_prod(a[q], bv, p, ep);
                        two_sum(s, p, t, et);
                        s = t;
                        comp = comp + (et + ep);
                        abs_s += std::fabs(a[q]) * std::fabs(bv);
                    }
                    rowp(C, ii, lwC)[j] = s + comp;
                    if (absAB) rowp(absAB, ii, lwAbs)[j] = abs_s;
                }
            }
        });
    }
    pool()->run(tasks);
}
