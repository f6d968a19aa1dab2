// keq_plan.cu -- the launch side shared by the persistent step kernels:
// stepping, buffer rebinding, error bits, reset, spin limit and the phase
// trace of a keq_plan (implicit or HOLO).  Kernels of both kinds take
// (device header, swap_io) and run as one cooperative launch per time step.
#include <cuda_runtime.h>
#include <stddef.h>
#include <string.h>

#include "keq_common.cuh"
#include "keq_internal.h"

namespace {
keq_status cuda_fail(cudaError_t e) {
    keq_internal_set_cuda_error(e);
    return KEQ_ERR_CUDA;
}
keq::PlanHead* head_of(keq_plan* plan) { return static_cast<keq::PlanHead*>(plan->dev); }
}  // namespace

extern "C" {

keq_status keq_plan_set_buffers(keq_plan* plan, const double* const* f_in, double* const* f_out,
                                keq_stream_t stream) {
    if (!plan || !f_in || !f_out) return KEQ_ERR_INVALID;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    for (int b = 0; b < plan->n_inst; ++b)
        if (!f_in[b] || !f_out[b] || f_in[b] == f_out[b]) return KEQ_ERR_INVALID;
    for (int b = 0; b < plan->n_inst; ++b) {
        unsigned char* rec = plan->host_inst.data() + (size_t)b * plan->inst_bytes;
        memcpy(rec + plan->off_f_in, &f_in[b], sizeof(void*));
        memcpy(rec + plan->off_f_out, &f_out[b], sizeof(void*));
    }
    cudaError_t e = cudaMemcpyAsync(plan->dev_inst, plan->host_inst.data(),
                                    plan->inst_bytes * plan->n_inst, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? KEQ_OK : cuda_fail(e);
}

keq_status keq_plan_step(keq_plan* plan, int32_t n_steps, int32_t parity, keq_stream_t stream) {
    if (!plan || n_steps < 0) return KEQ_ERR_INVALID;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (cudaSetDevice(plan->device) != cudaSuccess) return cuda_fail(cudaGetLastError());
    for (int k = 0; k < n_steps; ++k) {
        int swap_io = ((parity + k) & 1);
        // fresh barrier counter and error word for this launch (bar.count, err)
        cudaError_t e = cudaMemsetAsync(plan->dev, 0, offsetof(keq::PlanHead, err_sticky), s);
        if (e != cudaSuccess) return cuda_fail(e);
        void* args[] = {&plan->dev, &swap_io};
        e = cudaLaunchCooperativeKernel(plan->kernel, dim3(plan->grid), dim3(plan->threads), args,
                                        plan->smem, s);
        if (e != cudaSuccess) return cuda_fail(e);
    }
    return KEQ_OK;
}

void keq_plan_destroy(keq_plan* plan) { delete plan; }

keq_status keq_plan_set_trace(keq_plan* plan, unsigned long long* trace, int32_t iters,
                              keq_stream_t stream) {
    if (!plan || iters < 0 || (iters > 0 && !trace)) return KEQ_ERR_INVALID;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    keq::PlanHead* d = head_of(plan);
    unsigned long long* tp = iters > 0 ? trace : nullptr;
    cudaError_t e = cudaMemcpyAsync(&d->trace, &tp, sizeof(tp), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&d->trace_iters, &iters, sizeof(int), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? KEQ_OK : cuda_fail(e);
}

keq_status keq_plan_error(keq_plan* plan, keq_stream_t stream, int32_t* err_bits) {
    if (!plan || !err_bits) return KEQ_ERR_INVALID;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int v = 0;
    cudaError_t e = cudaMemcpyAsync(&v, &head_of(plan)->err_sticky, sizeof(int),
                                    cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e);
    *err_bits = v;
    return KEQ_OK;
}

keq_status keq_plan_reset(keq_plan* plan, keq_stream_t stream) {
    if (!plan) return KEQ_ERR_INVALID;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(plan->dev, 0, offsetof(keq::PlanHead, spin_limit), s);
    return e == cudaSuccess ? KEQ_OK : cuda_fail(e);
}

keq_status keq_plan_set_spin_limit(keq_plan* plan, unsigned long long limit, keq_stream_t stream) {
    if (!plan) return KEQ_ERR_INVALID;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const unsigned long long v = limit;
    cudaError_t e =
        cudaMemcpyAsync(&head_of(plan)->spin_limit, &v, sizeof(v), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? KEQ_OK : cuda_fail(e);
}

}  // extern "C"

// Grid size of a plan's cooperative launch: every resident CTA of the kernel.
keq_status keq_internal_plan_grid(keq_plan* plan) {
    int dev_id = 0, sms = 0, occ = 0;
    cudaGetDevice(&dev_id);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev_id);
    cudaError_t e = cudaFuncSetAttribute(plan->kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)plan->smem);
    if (e != cudaSuccess) return cuda_fail(e);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, plan->kernel, plan->threads, plan->smem);
    if (e != cudaSuccess) return cuda_fail(e);
    if (occ < 1 || sms < 1) return KEQ_ERR_UNSUPPORTED;
    plan->grid = sms * occ;
    return KEQ_OK;
}
