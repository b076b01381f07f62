// Launchers of the device kernels, called by the C ABI (api.cu).
#pragma once

#include <cuda_runtime.h>

#include "device_common.cuh"
#include "qs_internal.h"

namespace qs {

// Process-wide count of kernels this library launched (qs_launch_count).
void count_launches(int n);

cudaError_t launch_scale(int T, const Operands &op, const double *beta, int beta_case, int mfast,
                         cudaStream_t st);
cudaError_t launch_direct(int T, const Operands &op, const double *alpha, const double *beta,
                          int beta_case, int a_mfast, int b_nfast, cudaStream_t st);
cudaError_t launch_dot(int T, const Operands &op, const double *alpha, const double *beta,
                       int beta_case, cudaStream_t st);
cudaError_t launch_outer(int T, const Operands &op, const double *alpha, const double *beta,
                         int beta_case, int mfast, cudaStream_t st);

}  // namespace qs
