// Tensor-core paths: placeholder until the kernels land.
#include "kernels.h"
#include "tc.h"

namespace qs {

int tc_auto_method(const qs_plan *) { return QS_METHOD_NATIVE; }
void tc_geometry(qs_plan *) {}
int tc_prepare(qs_plan *) { return fail(QS_ENOTSUP, "tensor-core path not built"); }
int tc_execute(qs_plan *, const double *, const double *, int, cudaStream_t) {
  return fail(QS_ENOTSUP, "tensor-core path not built");
}
int tc_execute_grouped(int n, qs_plan *const *plans, const double *alpha, const double *beta,
                       cudaStream_t st) {
  for (int i = 0; i < n; ++i) {
    int rc = qs_execute(plans[i], alpha + 2 * i, beta + 2 * i, (void *)st);
    if (rc) return rc;
  }
  return QS_OK;
}

}  // namespace qs
