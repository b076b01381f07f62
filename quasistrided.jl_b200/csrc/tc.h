// Tensor-core paths (Ozaki INT8 slices, split-BF16x3) and grouped execution.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "qs_internal.h"

namespace qs {

// Method the autotuner picks for a nest-path plan with method AUTO.
int tc_auto_method(const qs_plan *p);
// Padded geometry of the packed panels (host only; no allocation).
void tc_geometry(qs_plan *p);
// Geometry + device workspace for the packed panels.
int tc_prepare(qs_plan *p);
// Pack + tensor-core GEMM + epilogue, enqueued on st.
// `ev` (nullable) receives an event before the first launch and after each.
int tc_execute(qs_plan *p, const double *alpha, const double *beta, int beta_case,
               cudaStream_t st, cudaEvent_t *ev = nullptr);
// Kernel class of a tensor-core plan in a grouped launch: plans of one class
// share every launch of the class (pack, GEMM, fixup).
enum { TC_CLASS_OZ6 = 0, TC_CLASS_OZ7 = 1, TC_CLASS_I8 = 2, TC_CLASS_BF16 = 3, TC_CLASS_OZ4 = 4, TC_NCLASS = 5 };
int tc_group_class(const qs_plan *p);

// The device tables of one class of a grouped launch: a host image built by
// tc_group_build and a device copy uploaded by tc_group_upload.
struct TcGroup {
  int cls = 0;
  std::vector<qs_plan *> plans;  // cost-descending
  std::vector<int> idx;          // position of each plan in the group's alpha/beta arrays
  std::vector<uint8_t> image;
  void *dev = nullptr;
  size_t dev_bytes = 0;
  size_t off_pack = 0, off_gemm = 0, off_tiles = 0, off_zero = 0, off_fix = 0, off_jobmap = 0, off_tilemap = 0;
  int njobs = 0, pack_blocks = 0, tiles = 0;
  int pack_kind = 2;       // element kind of the pack passes (tc.cu kPack*)
  std::vector<int> chunks;  // Ozaki pack chunks: block boundaries, first 0, last pack_blocks
  // Ozaki: the digit passes run on `aux`, chunk c after its row maxima
  // (event ev[c] on the launch stream), joined back through `join`.
  cudaStream_t aux = nullptr;
  std::vector<cudaEvent_t> ev;
  cudaEvent_t join = nullptr;
};
// alpha/beta hold 2 doubles per plan of the group, bcase one int per plan.
int tc_group_build(TcGroup &g, const double *alpha, const double *beta, const int *bcase);
int tc_group_upload(TcGroup &g, cudaStream_t st);
// Enqueues the class's launches; adds their count to *launches.
int tc_group_launch(const TcGroup &g, cudaStream_t st, int *launches);
// Frees the tables on `rel`, a stream already ordered after their last use.
void tc_group_release(TcGroup &g, cudaStream_t rel);

}  // namespace qs
