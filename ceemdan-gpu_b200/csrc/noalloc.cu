// Tridiagonal solve that allocates no memory.
//
// ceemdan_tridiag_f64 allocates its scratch (a copy of the systems and the workspace of the
// deeper partition levels) from the device allocator on every call.  Some callers cannot do
// that: real-time or signal-processing loops that forbid allocator calls (an allocation can
// synchronise the device and take unbounded time), hosts that pre-reserve all device memory
// for themselves, and plugins of frameworks whose memory pools must not be bypassed.
// ceemdan_tridiag_noalloc_f64 serves them: the scratch is a fixed array in the library's own
// device image.
//
// Costs and limits of that choice:
//   - the array (kNoallocScratchDoubles doubles, 8 MiB) is reserved on a device when the
//     library's device code is loaded there.  With lazy module loading (the CUDA default) that
//     happens at the first call on the device, so that first call may itself allocate those
//     8 MiB; later calls allocate nothing.  The memory stays reserved until the process exits;
//   - batch * (5 * n + 64) must not exceed kNoallocScratchDoubles; larger requests are
//     rejected with CEEMDAN_ERR_INVALID_ARG before anything is launched;
//   - all calls share the one array: two calls whose kernels overlap on the GPU (different
//     streams, or different host threads) race on it and corrupt each other's results;
//   - nothing in the array has to start at zero: every call writes each scratch element it
//     later reads, so the contents a previous call left behind are never used;
//   - the device address of the array is looked up (cudaGetSymbolAddress) by the first call
//     on each device and kept for the process; make that first call before starting any
//     stream capture.  A cudaDeviceReset of that device invalidates the kept address, so
//     this entry point must not be used on a device after it was reset;
//   - the call is synchronous, like ceemdan_tridiag_f64: it waits for its stream.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/ceemdan_b200.h"
#include "kernels.h"

namespace ceemdan {

// engine.cu: last-error text of the calling thread
void set_last_error(const std::string& what);

namespace {

constexpr size_t kNoallocScratchDoubles = (size_t)1 << 20;  // 8 MiB
constexpr int kMaxDevices = 64;

// File-scope scratch of the no-allocation entry point.  In host code this name only stands
// for the symbol; the device address comes from cudaGetSymbolAddress.
static __device__ __align__(256) double g_noalloc_scratch[kNoallocScratchDoubles];

std::mutex g_noalloc_mu;
double* g_noalloc_ptr[kMaxDevices] = {};

ceemdan_status noalloc_scratch(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_last_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
        return CEEMDAN_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        set_last_error("device ordinal beyond the no-allocation scratch table");
        return CEEMDAN_ERR_INVALID_ARG;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_last_error(std::string("cudaGetSymbolAddress(no-allocation scratch): ") +
                           cudaGetErrorString(e));
            return CEEMDAN_ERR_CUDA;
        }
        g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return CEEMDAN_OK;
}

}  // namespace
}  // namespace ceemdan

using namespace ceemdan;

extern "C" ceemdan_status ceemdan_tridiag_noalloc_f64(size_t batch, size_t n, const double* d_l,
                                                      const double* d_m, const double* d_u,
                                                      const double* d_r, double* d_x,
                                                      void* stream) {
    if (batch < 1 || n < 1 || batch > 65535 || !d_l || !d_m || !d_u || !d_r || !d_x) {
        set_last_error("invalid argument");
        return CEEMDAN_ERR_INVALID_ARG;
    }
    const size_t ws_stride = n + 64;
    if (n > kNoallocScratchDoubles || batch * (4 * n + ws_stride) > kNoallocScratchDoubles) {
        set_last_error("ceemdan_tridiag_noalloc_f64: batch*(5*n+64) = " +
                       std::to_string(batch * (4 * n + ws_stride)) +
                       " doubles exceeds the 1048576-double (8 MiB) static scratch");
        return CEEMDAN_ERR_INVALID_ARG;
    }
    double* scratch = nullptr;
    ceemdan_status s = noalloc_scratch(&scratch);
    if (s != CEEMDAN_OK) return s;
    cudaStream_t st = (cudaStream_t)stream;
    double* sys = scratch;
    double* ws = scratch + batch * 4 * n;
    k_tridiag_batched<<<(unsigned)batch, kTridiagThreads, 0, st>>>((int)n, d_l, d_m, d_u, d_r,
                                                                   d_x, sys, ws, ws_stride);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        set_last_error(std::string("ceemdan_tridiag_noalloc_f64: ") + cudaGetErrorString(e));
        return CEEMDAN_ERR_CUDA;
    }
    return CEEMDAN_OK;
}
