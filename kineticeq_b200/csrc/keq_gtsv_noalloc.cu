// keq_gtsv_noalloc.cu -- the batched tridiagonal solve with its scratch in a
// fixed device array of this library, for callers that cannot allocate
// device memory.
//
// Who needs it: a host runtime that hands this library only the tensors of
// the operation itself -- no workspace slot in its binding, and no device
// allocator it is allowed to call (for example a caller whose memory is all
// owned by a fixed pool of another runtime, or code that must not call
// cudaMalloc because that call can synchronise the whole device).  Such a
// caller cannot provide the scratch that keq_gtsv_strided_inplace asks for.
//
// The scratch is g_gtsv_scratch below: KEQ_GTSV_NOALLOC_MAX_ELEMS doubles
// (16 MiB), present on every GPU that loads the library until the process
// exits.  Host code cannot use the name g_gtsv_scratch as a device address
// (on the host it names a shadow variable), so the device address is looked
// up with cudaGetSymbolAddress once per device, with that device current, on
// the first call made on it, and cached.
#include <cuda_runtime.h>

#include <mutex>

#include "keq_internal.h"

namespace {

__device__ __align__(256) double g_gtsv_scratch[KEQ_GTSV_NOALLOC_MAX_ELEMS];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of g_gtsv_scratch on the current device (looked up once).
keq_status scratch_for_current_device(double** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        keq_internal_set_cuda_error(e);
        return KEQ_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) return KEQ_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_mu);
    if (g_scratch_addr[dev] == nullptr) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_gtsv_scratch);
        if (e != cudaSuccess || p == nullptr) {
            keq_internal_set_cuda_error(e != cudaSuccess ? e : cudaErrorInvalidSymbol);
            return KEQ_ERR_CUDA;
        }
        g_scratch_addr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_addr[dev];
    return KEQ_OK;
}

}  // namespace

extern "C" {

keq_status keq_gtsv_strided_inplace_noalloc(const double* dl, const double* d, const double* du,
                                            double* B, int32_t n, int32_t batch,
                                            keq_stream_t stream) {
    if (n < 0 || batch < 0) return KEQ_ERR_INVALID;
    if (n == 0 || batch == 0) return KEQ_OK;
    if (!dl || !d || !du || !B) return KEQ_ERR_INVALID;
    if ((long long)n * (long long)batch > (long long)KEQ_GTSV_NOALLOC_MAX_ELEMS)
        return KEQ_ERR_CAPACITY;
    double* scratch = nullptr;
    const keq_status st = scratch_for_current_device(&scratch);
    if (st != KEQ_OK) return st;
    // Every scratch element the kernel reads is written earlier in the same
    // call (the modified diagonal of its own system), so nothing is cleared.
    keq::gtsv_kernel<<<(batch + 127) / 128, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        dl, d, du, B, n, batch, scratch);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        keq_internal_set_cuda_error(e);
        return KEQ_ERR_CUDA;
    }
    return KEQ_OK;
}

}  // extern "C"
