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
  int shape = 0;                 // native shape (native_shape_for numbering) of every member
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

// Native-method tile shapes, as stored in a plan (qs_plan_info.native_tile
// is the shape + 1): 0-3 the SIMT gather GEMM's tiles (direct_shape
// numbering), 4 + s the DMMA kernel's tile s (0: 128x128, 1: 128x64,
// 2: 64x64, 3: 128x32, 4: 256x16, 5: 128x128 with 16 warps), for real
// Float64 operands only.
constexpr int kSimtShapes = 4, kDmmaShapes = 6, kNativeShapes = kSimtShapes + kDmmaShapes;
// The shape for compute type T with operand eltypes TA, TB: native_tile
// (1..kNativeShapes) if it applies, else by M and N (grouped: by N only,
// since the group's other problems fill the GPU).  Skinny problems (the
// read-B-in-place kernel's N <= 16, K <= 64) keep the SIMT numbering.
int native_shape_for(int T, int TA, int TB, int64_t M, int64_t N, int64_t K, int native_tile, bool grouped);

// DMMA (mma.sync .f64) gather GEMM: real Float64 A and B, any real C.
bool dmma_eligible(int T, int TA, int TB);
int dmma_shape_mn(int64_t M, int64_t N);
int dmma_shape_n(int64_t N);
void dmma_tile_dims(int shape, int *bm, int *bn);
cudaError_t launch_dmma(const Operands &op, const double *alpha, const double *beta, int beta_case,
                        int a_mfast, int b_nfast, int shape, cudaStream_t st);
cudaError_t dmma_group_launch(int shape, const void *jobs, int njobs, int blocks, cudaStream_t st);

// The operands of a plan as the kernels read them.
Operands make_operands(const qs_plan *p);
// Zero (0), One (1) or general (2) after conversion to compute type T.
int scalar_case(int T, const double *v);

}  // namespace qs
