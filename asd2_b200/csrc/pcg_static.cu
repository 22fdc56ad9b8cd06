// Jacobi-PCG on a caller-assembled GFM system that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host application that owns all
// device memory through its own pool allocator and hands plug-ins only
// pre-registered buffers, code on a latency-critical path where cudaMalloc /
// cudaFree would implicitly synchronise the device, or a process that has
// already reserved the whole GPU.  For them asd2g_pcg_solve_static keeps the
// solver's work space (r, two direction vectors, q, the inverse diagonal,
// the reduction partials and the solver scalars) in one file-scope
// __device__ array of fixed size, so the caller only passes the system and
// the output vector.
//
// Properties a caller must know:
//  * Capacity: at most ASD2G_STATIC_MAX_UNKNOWNS (512 * 512) unknowns; larger
//    systems are rejected with ASD2G_E_ARG.  The array (about 10 MiB) is held
//    on every GPU that loads the library until the process exits.
//  * Set-up: the first call on a device resolves the array's device address
//    (cudaGetSymbolAddress, with that device current) and caches it, so make
//    that first call before any stream capture begins.  Later calls look
//    the address up again unless their stream is capturing, so the cached
//    address follows a cudaDeviceReset or another context made current on
//    the device.
//  * Sharing: every call on a device uses the same array and leaves its last
//    contents behind.  Calls that overlap on the GPU (different streams or
//    host threads at the same time) race on it and must be serialised by the
//    caller.  Each call re-initialises everything it reads before reading it
//    (the solver scalars, including the reduction ticket counter, are reset
//    first).
#include <mutex>

#include "asd2g.h"
#include "pressure.cuh"

namespace asd2g {
int api_exception(const char *fn);  // the entry points' exception handler (api.cu)
}  // namespace asd2g

namespace asd2g {
namespace {

constexpr int64_t kMaxUnknowns = ASD2G_STATIC_MAX_UNKNOWNS;
constexpr size_t kStateDoubles = (sizeof(KState) + sizeof(double) - 1) / sizeof(double);
// [minv | r | p_a | p_b | q] (kMaxUnknowns each) | partials | KState
constexpr size_t kScratchDoubles = 5 * (size_t)kMaxUnknowns + 3 * (size_t)RED_BLOCKS_MAX + kStateDoubles;

__device__ __align__(256) double g_pcg_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
double *g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

// Inverse diagonal for the Jacobi preconditioner (InvertMatrixDiagonal,
// poisson2d.cpp:577-585); the pinned cell keeps 0 so it never moves.
__global__ void k_static_minv(int64_t n, int pinned, const double *__restrict__ diag, double *__restrict__ minv) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        minv[k] = (pinned && k == 0) ? 0.0 : 1.0 / diag[k];
}

int static_fail(int code, const char *msg) {
    asd2g_set_error_text(msg);
    return code;
}

}  // namespace
}  // namespace asd2g

using namespace asd2g;

extern "C" int asd2g_pcg_solve_static(int nx, int ny, int pinned, const double *diag, const double *ce,
                                      const double *cn, const double *b, double *x, double tol, int maxit,
                                      void *stream, int *iters, double *rel_resid) try {
    if (nx < 1 || ny < 1) return static_fail(ASD2G_E_ARG, "asd2g_pcg_solve_static: nx and ny must be positive");
    if ((int64_t)nx * ny > kMaxUnknowns)
        return static_fail(ASD2G_E_ARG,
                           "asd2g_pcg_solve_static: system exceeds the fixed work space of "
                           "ASD2G_STATIC_MAX_UNKNOWNS = 262144 unknowns (512 x 512)");
    if (!diag || !ce || !cn || !b || !x) return static_fail(ASD2G_E_ARG, "asd2g_pcg_solve_static: null pointer");
    if (maxit < 0) return static_fail(ASD2G_E_ARG, "asd2g_pcg_solve_static: maxit must be >= 0");
    // An error left pending by earlier work of the caller is reported as such,
    // not blamed on this call's launches.
    if (cudaGetLastError() != cudaSuccess)
        return static_fail(ASD2G_E_CUDA, "asd2g_pcg_solve_static: a CUDA error was pending before the call");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return static_fail(ASD2G_E_CUDA, "asd2g_pcg_solve_static: no current CUDA device");
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) {
        cudaGetLastError();
        return static_fail(ASD2G_E_CUDA, "asd2g_pcg_solve_static: invalid stream");
    }
    double *base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_scratch_mu);
        // Looked up on every uncaptured call (cheap): a cudaDeviceReset or
        // another context current on this device moves the array.
        if (!g_scratch_addr[dev] || cap == cudaStreamCaptureStatusNone) {
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_pcg_scratch);
            if (e != cudaSuccess || !p) {
                cudaGetLastError();
                g_scratch_addr[dev] = nullptr;
                return static_fail(ASD2G_E_CUDA, "asd2g_pcg_solve_static: cudaGetSymbolAddress failed");
            }
            g_scratch_addr[dev] = static_cast<double *>(p);
        }
        base = g_scratch_addr[dev];
    }
    const int64_t n = (int64_t)nx * ny;
    double *minv = base, *r = base + kMaxUnknowns, *pa = base + 2 * kMaxUnknowns, *pb = base + 3 * kMaxUnknowns,
           *q = base + 4 * kMaxUnknowns, *partial = base + 5 * kMaxUnknowns;
    KState *ks = reinterpret_cast<KState *>(partial + 3 * RED_BLOCKS_MAX);
    Sys S{const_cast<double *>(diag), nullptr, const_cast<double *>(ce), nullptr, const_cast<double *>(cn), minv,
          const_cast<double *>(b), pinned ? 1 : 0};
    Grid g{};
    g.nx = nx;
    g.ny = ny;
    k_static_minv<<<red_blocks(n), 256, 0, st>>>(n, S.pinned, diag, minv);
    launch_set_kstate(ks, tol, maxit, 0, 0.0, st);
    launch_pcg_init(g, S, x, r, pa, ks, partial, st);
    if (cudaGetLastError() != cudaSuccess) return static_fail(ASD2G_E_CUDA, "asd2g_pcg_solve_static: launch failed");
    // Iterations go in pairs (the direction vectors alternate); each one
    // returns at entry once the solver scalars say done.  Chunks of up to 64
    // iterations are launched between host checks, the last one cut so that
    // no more than maxit (rounded up to even) iterations are launched.
    const int64_t chunk = 64;
    KState hk{};
    for (int64_t launched = 0;;) {
        const int64_t left = (int64_t)maxit - launched;
        const int64_t now = left < chunk ? left : chunk;
        for (int64_t k = 0; k < now; k += 2) {
            launch_pcg_iter(g, S, x, r, pa, pb, q, ks, partial, st);
            launch_pcg_iter(g, S, x, r, pb, pa, q, ks, partial, st);
        }
        launched += now + (now & 1);
        if (cudaGetLastError() != cudaSuccess)
            return static_fail(ASD2G_E_CUDA, "asd2g_pcg_solve_static: launch failed");
        if (cudaMemcpyAsync(&hk, ks, sizeof(KState), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            cudaGetLastError();
            return static_fail(ASD2G_E_CUDA, "asd2g_pcg_solve_static: CUDA error during the solve");
        }
        if (hk.done || launched >= (int64_t)maxit) break;
    }
    if (iters) *iters = hk.it;
    if (rel_resid) *rel_resid = hk.res;
    if (hk.status == -5) return static_fail(ASD2G_E_NONFINITE, "asd2g_pcg_solve_static: non-finite residual");
    if (hk.status == -6) return static_fail(ASD2G_E_BREAKDOWN, "asd2g_pcg_solve_static: breakdown (p.Ap = 0)");
    return !(hk.res > tol) ? ASD2G_OK : ASD2G_NOT_CONVERGED;
} catch (...) {
    return asd2g::api_exception("asd2g_pcg_solve_static");
}
