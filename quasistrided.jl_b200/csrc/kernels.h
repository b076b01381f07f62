// Launchers of the device kernels, called by the C ABI (api.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "device_common.cuh"
#include "qs_internal.h"

namespace qs {

// Process-wide count of kernels this library launched (qs_launch_count).
void count_launches(int n);

cudaError_t launch_scale(int T, const Operands &op, const double *beta, int beta_case, int mfast,
                         cudaStream_t st);
cudaError_t launch_direct(int T, const Operands &op, const double *alpha, const double *beta,
                          int beta_case, int a_mfast, int b_nfast, int shape, cudaStream_t st);
cudaError_t launch_dot(int T, const Operands &op, const double *alpha, const double *beta,
                       int beta_case, cudaStream_t st);
cudaError_t launch_outer(int T, const Operands &op, const double *alpha, const double *beta,
                         int beta_case, int mfast, cudaStream_t st);

// Native (gather) GEMMs of many plans of one compute type as one launch.
struct NativeGroup {
  int T = 0;
  int shape = 0;                 // tile shape (direct_shape_mn numbering) of every member
  std::vector<qs_plan *> plans;  // K-descending
  std::vector<int> idx;          // position of each plan in the group's alpha/beta arrays
  std::vector<uint8_t> image;    // host image of the job table
  void *dev = nullptr;
  size_t dev_bytes = 0;
  int blocks = 0;
};
// ops[i] are the operands of plans[i]; alpha/beta hold 2 doubles per plan of
// the group, bcase one int per plan.
int native_group_build(NativeGroup &g, const Operands *ops, const double *alpha, const double *beta,
                       const int *bcase);
cudaError_t native_group_launch(const NativeGroup &g, cudaStream_t st);

// Tile shape of the gather GEMM for compute type T and N (0: 64x64,
// 1: 128x32, 2: 256x16; complex: 0 = 32x32).
int direct_shape(int T, int64_t N);
// The plan's choice: direct_shape, or 3 (32x32) when a 64x64 grid would not
// fill the GPU.
int direct_shape_mn(int T, int64_t M, int64_t N);

// The operands of a plan as the kernels read them.
Operands make_operands(const qs_plan *p);
// Zero (0), One (1) or general (2) after conversion to compute type T.
int scalar_case(int T, const double *v);

}  // namespace qs
