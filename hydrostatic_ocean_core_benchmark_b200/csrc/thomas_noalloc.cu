// Batched tridiagonal solve that allocates no device memory.
//
// oc_thomas obtains its elimination scratch (one coefficient per row and
// column) from cudaMallocAsync on every call. Some callers cannot allow that:
// a host model that reserves all its device memory at start-up and must keep a
// fixed footprint afterwards, or a pipeline of asynchronous work that cannot
// tolerate the device-wide synchronisation cudaMalloc/cudaFree may perform.
// oc_thomas_noalloc gives them the same solve with the scratch in a fixed
// array of this library instead.
//
// The scratch is a file-scope __device__ array of OC_THOMAS_NOALLOC_MAX_CELLS
// doubles (8 MiB). CUDA loads a library's device code lazily, so the array is
// committed on a device by the first call made with that device current, and
// that device then holds it until the process exits. That first call also
// takes the array's device address (cudaGetSymbolAddress) and keeps it for the
// device. A host that fixes its device footprint at start-up therefore makes
// one warm-up call per device at start-up; the same warm-up call has to come
// before any stream capture. The kept address belongs to the device's current
// context: after cudaDeviceReset the library must not be used again in the
// process. All calls share the one array and it keeps the last call's
// contents: calls whose work can overlap on the GPU (different streams, or
// several host threads) race on it and must be serialised by the caller.
// Every scratch element a solve reads is written earlier by the same solve,
// so nothing has to be cleared between calls.

#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "ocean_b200.h"
#include "step_kernels.cuh"

namespace {

static __device__ __align__(256) double g_noalloc_scratch[OC_THOMAS_NOALLOC_MAX_CELLS];

constexpr int kMaxDevices = 64;
double* g_scratch_ptr[kMaxDevices] = {};
std::mutex g_setup_lock;

// device address of the scratch for the current device, looked up once
int scratch_for_current_device(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return OC_ERR_CUDA;
    if (dev < 0 || dev >= kMaxDevices) return OC_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> guard(g_setup_lock);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            std::fprintf(stderr, "oc_thomas_noalloc: cudaGetSymbolAddress failed on device %d: %s\n", dev,
                         cudaGetErrorString(e));
            return OC_ERR_CUDA;
        }
        g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_ptr[dev];
    return OC_OK;
}

}  // namespace

extern "C" int oc_thomas_noalloc(const double* sub, const double* diag, const double* sup,
                                 const double* rhs, double* x, int32_t n, int32_t ncols, void* stream) {
    if (!sub || !diag || !sup || !rhs || !x || n < 1 || ncols < 1) return OC_ERR_ARG;
    const long long cells = (long long)n * (long long)ncols;
    if (cells > OC_THOMAS_NOALLOC_MAX_CELLS) {
        std::fprintf(stderr,
                     "oc_thomas_noalloc: %d rows x %d columns = %lld cells exceed the fixed scratch of "
                     "%d cells; use oc_thomas\n",
                     n, ncols, cells, OC_THOMAS_NOALLOC_MAX_CELLS);
        return OC_ERR_TOO_LARGE;
    }
    // an error left pending by the caller's own earlier work is not this
    // solve's: report it without consuming it, so the caller's check still sees it
    if (cudaPeekAtLastError() != cudaSuccess) return OC_ERR_CUDA;
    double* scratch = nullptr;
    const int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    oc::launch_thomas(sub, diag, sup, rhs, x, scratch, n, ncols, (cudaStream_t)stream);
    return cudaGetLastError() == cudaSuccess ? OC_OK : OC_ERR_CUDA;
}
