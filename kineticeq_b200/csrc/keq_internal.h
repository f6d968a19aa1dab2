// keq_internal.h -- host-side helpers shared by the library's .cu files.
#pragma once

#include <cuda_runtime.h>

#include "../../include/keq_b200.h"

// Remember the last CUDA error of the calling thread for keq_last_cuda_error().
void keq_internal_set_cuda_error(cudaError_t e);
