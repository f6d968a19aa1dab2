// keq_internal.h -- host-side helpers shared by the library's .cu files.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "../../include/keq_b200.h"

// Remember the last CUDA error of the calling thread for keq_last_cuda_error().
void keq_internal_set_cuda_error(cudaError_t e);

// Host object behind the opaque keq_plan of the C ABI, shared by the
// persistent step kernels (implicit and HOLO).  The device header `dev`
// starts with a keq::PlanHead; instance records are `inst_bytes` each and
// hold their f_in / f_out pointers at the given byte offsets.
enum { KEQ_PLAN_IMPLICIT = 0, KEQ_PLAN_HOLO = 1 };
struct keq_plan {
    int kind;
    void* dev;
    void* dev_inst;
    std::vector<unsigned char> host_inst;
    size_t inst_bytes;
    size_t off_f_in, off_f_out;
    const void* kernel;
    size_t smem;
    int threads;
    int grid;
    int n_inst;
    int device;
};

// Sets plan->grid to every resident CTA of plan->kernel (occupancy query).
keq_status keq_internal_plan_grid(keq_plan* plan);

namespace keq {
// Batched tridiagonal solve (keq_kernels.cu): one thread per system; cp is
// n * batch doubles of scratch that every call overwrites before reading.
__global__ void __launch_bounds__(128) gtsv_kernel(const double* __restrict__ dl,
                                                   const double* __restrict__ d,
                                                   const double* __restrict__ du,
                                                   double* __restrict__ B, int n, int batch,
                                                   double* __restrict__ cp);
}  // namespace keq
