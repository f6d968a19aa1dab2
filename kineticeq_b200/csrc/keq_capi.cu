// keq_capi.cu -- version, status strings and error bookkeeping of the C ABI.
#include <cuda_runtime.h>

#include "keq_internal.h"

namespace {
thread_local char g_last_cuda_error[256] = {0};
}

void keq_internal_set_cuda_error(cudaError_t e) {
    const char* s = cudaGetErrorString(e);
    int i = 0;
    for (; s && s[i] && i < 255; ++i) g_last_cuda_error[i] = s[i];
    g_last_cuda_error[i] = 0;
}

extern "C" {

int32_t keq_abi_version(void) { return 1; }

const char* keq_status_string(int32_t status) {
    switch (status) {
        case KEQ_OK: return "ok";
        case KEQ_ERR_INVALID: return "invalid argument";
        case KEQ_ERR_WORKSPACE: return "workspace too small or misaligned";
        case KEQ_ERR_CUDA: return "CUDA runtime error";
        case KEQ_ERR_TIMEOUT: return "device-side wait timed out";
        case KEQ_ERR_NONFINITE: return "NaN/Inf detected in f_tmp";
        case KEQ_ERR_NOCONV: return "iteration cap reached without convergence";
        case KEQ_ERR_UNSUPPORTED: return "unsupported device or configuration";
        case KEQ_ERR_CAPACITY: return "request exceeds the fixed capacity of this entry point";
        default: return "unknown status";
    }
}

const char* keq_last_cuda_error(void) { return g_last_cuda_error; }

}  // extern "C"
