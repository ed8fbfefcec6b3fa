// noalloc.cu -- an LU solve for callers that cannot allocate device memory.
//
// Some callers must not allocate: a host program whose memory manager owns every device
// allocation and forbids any other, or a real-time loop with a fixed memory budget that may not
// grow.  b2m_dev_MatrixLinEQSolveNoAlloc serves them: the caller
// passes device inputs and outputs, and every intermediate (the LU factors, pivots, permutation,
// right-hand-side buffers and status words) lives in one file-scope device array of fixed size.
// The call makes no cudaMalloc / cudaFree and uses no context workspace.
#include <mutex>

#include "common.cuh"
#include "kernels.cuh"

namespace b2m {
namespace {

constexpr int64_t kNaMaxN = 512;     // largest order accepted
constexpr int64_t kNaMaxRhs = 64;    // largest number of right-hand sides accepted
constexpr int64_t kNaLd = kNaMaxN;   // row stride of the factor buffer (elements)
constexpr int64_t kNaLdx = kNaMaxRhs;
constexpr int64_t kNaLuDoubles = kNaMaxN * kNaLd;
constexpr int64_t kNaXDoubles = kNaMaxN * kNaLdx;
constexpr int64_t kNaIntDoubles = 1024;  // pivots, permutation and status words (int32)
constexpr int64_t kNaDoubles = kNaLuDoubles + 2 * kNaXDoubles + kNaIntDoubles;  // 2.5 MiB + 8 KiB

// Shared by every call on a device; it keeps the last call's contents.
static __device__ __align__(256) double g_noalloc_scratch[kNaDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_na_mutex;
double* g_na_base[kMaxDevices] = {};  // device address of g_noalloc_scratch, per device

}  // namespace
}  // namespace b2m

using namespace b2m;

extern "C" int32_t b2m_dev_MatrixLinEQSolveNoAlloc(void* stream, const double* A, int64_t LineWidthA, int64_t width,
                                                   const double* B, int64_t LineWidthB, double* X,
                                                   int64_t LineWidthX, int64_t Width2, int32_t* status) {
    if (!A || !B || !X) return B2M_ERR_ARG;
    if (width <= 0 || Width2 <= 0 || LineWidthA < width * 8 || (LineWidthA % 8) || LineWidthB < Width2 * 8 ||
        (LineWidthB % 8) || LineWidthX < Width2 * 8 || (LineWidthX % 8))
        return B2M_ERR_DIM;
    if (width > kNaMaxN || Width2 > kNaMaxRhs) return B2M_ERR_UNSUPPORTED;  // beyond the fixed scratch
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return B2M_ERR_CUDA;
    double* base = nullptr;
    {
        // one-time set-up per device, with that device current: host code cannot use the
        // symbol itself (it is a host-side stand-in), only the address the runtime reports
        std::lock_guard<std::mutex> lk(g_na_mutex);
        if (!g_na_base[dev]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
                cudaGetLastError();
                return B2M_ERR_CUDA;
            }
            g_na_base[dev] = static_cast<double*>(p);
        }
        base = g_na_base[dev];
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    double* LU = base;
    double* Xs = LU + kNaLuDoubles;
    double* T = Xs + kNaXDoubles;
    int32_t* ints = reinterpret_cast<int32_t*>(T + kNaXDoubles);
    int32_t* ipiv = ints;
    int32_t* perm = ints + kNaMaxN;
    int32_t* words = ints + 2 * kNaMaxN;

    // a context on the stack: it points at the scratch status words and never touches the
    // workspace allocator
    Ctx c;
    c.device = dev;
    c.stream = st;
    c.own_stream = st;
    c.d_status = words;
    c.use_graphs = false;  // instantiating a graph may allocate; this path launches directly
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess) c.smem_optin = v;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess) c.num_sms = v;

    const int64_t n = width, k = Width2;
    // what must start at zero: the status words and the pivot vector
    if (cudaMemsetAsync(words, 0, kNumStatus * sizeof(int32_t), st) != cudaSuccess) return B2M_ERR_CUDA;
    if (cudaMemsetAsync(ipiv, 0, (size_t)n * sizeof(int32_t), st) != cudaSuccess) return B2M_ERR_CUDA;
    B2M_TRY(copy_matrix(&c, st, LU, kNaLd * 8, A, LineWidthA, n, n));
    B2M_TRY(lu_factor_f64(&c, st, LU, kNaLd, n, ipiv, perm));
    B2M_TRY(copy_matrix(&c, st, Xs, kNaLdx * 8, B, LineWidthB, n, k));
    B2M_TRY(lu_solve_f64(&c, st, LU, kNaLd, n, perm, Xs, kNaLdx, k, T));
    B2M_TRY(copy_matrix(&c, st, X, LineWidthX, Xs, kNaLdx * 8, n, k));
    // the caller's result word: leOk, leSingular, or B2M_ERR_TIMEOUT when a bounded wait in the panel
    // or the GEMM gave up (X is then unfinished)
    if (status) B2M_TRY(publish_status(&c, st, words, status));
    return B2M_OK;
}
