// Tensor-core paths (Ozaki INT8 slices, split-BF16x3) and grouped execution.
#pragma once

#include <cuda_runtime.h>

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
// Many independent plans as one launch per stage.
int tc_execute_grouped(int n, qs_plan *const *plans, const double *alpha, const double *beta,
                       cudaStream_t st);

}  // namespace qs
