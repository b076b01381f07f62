// qs_contract_noalloc: contract! through the gather kernels without any
// device allocation.
//
// Some callers cannot allocate device memory at the moment they contract:
// a serving loop that must not stall other in-flight requests (cudaMalloc
// and cudaFree synchronize the whole device), or a host runtime that owns
// the device's memory through its own pool and forbids raw allocations.
// This entry point plans on the host and keeps the only scratch the gather
// kernels need — the M/N/K offset tables — in one file-scope device array of
// fixed size instead of a per-plan workspace.  The caller still passes A, B
// and C.
//
// Limits and sharing:
//  - The scratch holds at most kNoAllocEntries int64 offsets; a contraction
//    needs 2 * (M + N + K) of them (two maps per group).  Larger problems
//    are rejected with QS_EINVAL before anything is launched.
//  - Every call on a device uses the same array and leaves its own tables in
//    it.  Each call rewrites every entry it reads before reading it, so
//    nothing needs clearing between calls; calls that overlap on the GPU
//    (different streams, or different host threads) race on the array.
//  - The array lives in every GPU that loads the library until the process
//    exits.
//  - The first call on each device looks the array's device address up
//    (cudaGetSymbolAddress) with that device current; make that first call
//    before any stream capture on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <sstream>

#include "kernels.h"
#include "qs_internal.h"

namespace qs {

constexpr int64_t kNoAllocEntries = int64_t(1) << 19;  // 4 MiB of int64 offsets

static __device__ __align__(256) int64_t g_noalloc_scratch[kNoAllocEntries];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
int64_t *g_scratch_ptr[kMaxDevices] = {};

// The array's device address for the current device, looked up once per
// device.  In host code the symbol itself is only a host-side stand-in.
int scratch_for_device(int dev, int64_t **out) {
  if (dev < 0 || dev >= kMaxDevices) return fail(QS_EINVAL, "ArgumentError: device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    int64_t *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || ptr == nullptr) {
      std::ostringstream s;
      s << "cudaGetSymbolAddress of the no-alloc scratch failed: " << cudaGetErrorString(e);
      return fail(QS_ECUDA, s.str());
    }
    g_scratch_ptr[dev] = ptr;
  }
  *out = g_scratch_ptr[dev];
  return QS_OK;
}

// The three groups' offset tables (mixed radix, first label fastest, as
// fill_offsets) written straight into the scratch: [M map0 | M map1 |
// N map0 | N map1 | K map0 | K map1].
struct FillArgs {
  Group g[3];
  int64_t len[3];
  int64_t *out;
};

__global__ void noalloc_fill_offsets(const __grid_constant__ FillArgs a) {
  const int64_t total = a.len[0] + a.len[1] + a.len[2];
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    int which = 0;
    int64_t q = e, base = 0;
    while (which < 2 && q >= a.len[which]) {
      q -= a.len[which];
      base += 2 * a.len[which];
      ++which;
    }
    const Group &g = a.g[which];
    int64_t r = q, o0 = 0, o1 = 0;
    for (int d = 0; d < g.D; ++d) {
      int64_t x = r % g.len[d];
      r /= g.len[d];
      o0 += x * g.st[0][d];
      o1 += x * g.st[1][d];
    }
    a.out[base + q] = o0;
    a.out[base + a.len[which] + q] = o1;
  }
}

}  // namespace
}  // namespace qs

using namespace qs;

extern "C" int qs_contract_noalloc(const qs_view *C, const double *alpha, const qs_view *A,
                                   const int64_t *indA, const qs_view *B, const int64_t *indB,
                                   const double *beta, const int64_t *indC,
                                   const qs_plan_options *opts, void *stream) {
  if (!alpha || !beta) return fail(QS_EINVAL, "ArgumentError: alpha/beta is NULL");
  qs_plan_options o{};
  if (opts) o = *opts;
  if (o.flags & QS_PLAN_BATCH_LABELS)
    return fail(QS_ENOTSUP, "ArgumentError: qs_contract_noalloc does not take batch labels");
  qs_plan p;  // host-side plan on the stack; no device workspace
  int rc = plan_host(&p, C, A, indA, B, indB, indC, &o);
  if (rc) return rc;
  if (!is_complex(p.T) && (alpha[1] != 0.0 || beta[1] != 0.0))
    return fail(QS_EINVAL, "InexactError: a complex alpha/beta does not convert to the real compute type");
  if (p.path == QS_PATH_EMPTY) return QS_OK;
  const int64_t need = 2 * (p.M + p.N + p.K);
  if (need > kNoAllocEntries) {
    std::ostringstream s;
    s << "ArgumentError: qs_contract_noalloc needs " << need << " offset entries (2*(M+N+K)); its "
      << "static scratch holds at most " << kNoAllocEntries << " — use qs_plan_contract/qs_execute";
    return fail(QS_EINVAL, s.str());
  }
  const int nt = o.native_tile;
  if (nt < 0 || nt > kNativeShapes) return fail(QS_EINVAL, "ArgumentError: native_tile must be 0..10");
  const int acase = scalar_case(p.T, alpha), bcase = scalar_case(p.T, beta);
  const bool scale_only = acase == 0 || p.path == QS_PATH_SCALE;
  if ((rc = check_bounds(&p, !scale_only))) return rc;
  if (scale_only && bcase == 1) return QS_OK;  // C *= 1: nothing to launch, as qs_execute
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(QS_ECUDA, "cudaGetDevice failed");
  int64_t *scratch = nullptr;
  if ((rc = scratch_for_device(dev, &scratch))) return rc;

  FillArgs f;
  f.g[0] = p.mg;
  f.g[1] = p.ng;
  f.g[2] = p.kg;
  f.len[0] = p.M;
  f.len[1] = p.N;
  f.len[2] = p.K;
  f.out = scratch;
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t total = p.M + p.N + p.K;
  int grid = (int)std::min<int64_t>((total + 255) / 256, 1184);
  if (grid < 1) grid = 1;
  noalloc_fill_offsets<<<grid, 256, 0, st>>>(f);

  Operands op;
  op.A = p.Adata;
  op.B = p.Bdata;
  op.C = p.Cdata;
  op.Abase = p.Abase;
  op.Bbase = p.Bbase;
  op.Cbase = p.Cbase;
  op.TA = p.TA;
  op.TB = p.TB;
  op.TC = p.TC;
  op.conjA = p.conjA;
  op.conjB = p.conjB;
  op.offMA = scratch;
  op.offMC = scratch + p.M;
  op.offNB = scratch + 2 * p.M;
  op.offNC = scratch + 2 * p.M + p.N;
  op.offKA = scratch + 2 * (p.M + p.N);
  op.offKB = scratch + 2 * (p.M + p.N) + p.K;
  op.M = p.M;
  op.N = p.N;
  op.K = p.K;
  if (scale_only) {
    e = launch_scale(p.T, op, beta, bcase, p.c_mfast, st);
  } else if (p.path == QS_PATH_DOT) {
    e = launch_dot(p.T, op, alpha, beta, bcase, st);
  } else if (p.path == QS_PATH_OUTER) {
    e = launch_outer(p.T, op, alpha, beta, bcase, p.c_mfast, st);
  } else {
    // The kernel and tile shape qs_plan_contract would give the same problem.
    const int shape = native_shape_for(p.T, p.TA, p.TB, p.M, p.N, p.K, nt, false);
    e = launch_direct(p.T, op, alpha, beta, bcase, p.a_mfast, p.b_nfast, shape, st);
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    std::ostringstream s;
    s << "CUDA error in qs_contract_noalloc: " << cudaGetErrorString(e);
    return fail(QS_ECUDA, s.str());
  }
  count_launches(2);  // the offset fill and one kernel
  return QS_OK;
}
