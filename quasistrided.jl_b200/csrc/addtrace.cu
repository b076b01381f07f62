// tensoradd! / tensortrace! on the device:
//   C[indC] = alpha * sum over the traced labels of op(A)[indA] + beta * C[indC]
// Every label of indC appears once in indA; every other label of indA appears
// exactly twice (a traced pair).  With no pairs this is TO.tensoradd!
// (permute and add); with pairs, TO.tensortrace!.  The reference has no
// kernel of its own for these and forwards them to StridedNative on the host
// (src/integrations/tensoroperations.jl:90-107); keeping them on the device
// lets whole @tensor networks stay there.
//
// One grid-stride kernel; the view geometry travels by value (no tables, no
// allocation).  Each thread decomposes its linear index of C (first label
// fastest) into the offsets of C and A; the traced offsets of A, when there
// are at most kTraceStage of them, are staged once per CTA in shared memory.
// Control semantics as execute!: beta == 0 never reads C, alpha == 0 never
// reads A, an empty C is a no-op, bounds are checked before any launch.
#include <cuda_runtime.h>

#include <cmath>
#include <sstream>
#include <string>

#include "device_common.cuh"
#include "kernels.h"
#include "qs_internal.h"

namespace qs {

constexpr int kAddMaxRank = 16;
constexpr int kTraceStage = 1024;

struct AddArgs {
  const void *A;
  void *C;
  int64_t Abase, Cbase;
  int TA, TC, conjA;
  int nc, nt;                    // free (C) dims and traced pairs
  int64_t csize[kAddMaxRank];    // C dims in indC order
  int64_t cstC[kAddMaxRank];     // their strides in C
  int64_t cstA[kAddMaxRank];     // and in A
  int64_t tsize[kAddMaxRank];    // traced pair extents
  int64_t tstA[kAddMaxRank];     // sum of the pair's two strides in A
  int64_t total;                 // elements of C
  int64_t tracelen;              // product of tsize
  int read_a;                    // 0 when alpha == 0
};

__device__ __forceinline__ int64_t trace_offset(const AddArgs &a, int64_t t) {
  int64_t off = 0;
  for (int d = 0; d < a.nt; ++d) {
    const int64_t q = t / a.tsize[d];
    off += (t - q * a.tsize[d]) * a.tstA[d];
    t = q;
  }
  return off;
}

template <class T>
__global__ void __launch_bounds__(256) add_trace_kernel(const __grid_constant__ AddArgs a, Scalars<T> s) {
  __shared__ int64_t sT[kTraceStage];
  const bool staged = a.tracelen <= kTraceStage;
  if (staged && a.read_a)
    for (int64_t t = threadIdx.x; t < a.tracelen; t += blockDim.x) sT[t] = trace_offset(a, t);
  __syncthreads();
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < a.total;
       e += (int64_t)gridDim.x * blockDim.x) {
    int64_t r = e, oc = 0, oa = 0;
    for (int d = 0; d < a.nc; ++d) {
      const int64_t q = r / a.csize[d];
      const int64_t i = r - q * a.csize[d];
      oc += i * a.cstC[d];
      oa += i * a.cstA[d];
      r = q;
    }
    T acc = tzero<T>();
    if (a.read_a) {
      const int64_t base = a.Abase + oa;
      for (int64_t t = 0; t < a.tracelen; ++t) {
        const int64_t to = staged ? sT[t] : trace_offset(a, t);
        const T x = Loader<T>::load(a.A, base + to, a.TA, a.conjA);
        if constexpr (is_cplx<T>::value) {
          acc.re += x.re;
          acc.im += x.im;
        } else {
          acc += x;
        }
      }
    }
    const int64_t idx = a.Cbase + oc;
    const T old = s.beta_case == 0 ? tzero<T>() : load_c<T>(a.C, idx, a.TC);
    store_c<T>(a.C, idx, a.TC, axpby(s, acc, old));
  }
}

template <class T>
static Scalars<T> add_scalars(const double *alpha, const double *beta, int beta_case) {
  Scalars<T> s;
  if constexpr (is_cplx<T>::value) {
    using R = typename real_of<T>::type;
    s.alpha.re = (R)alpha[0]; s.alpha.im = (R)alpha[1];
    s.beta.re = (R)beta[0]; s.beta.im = (R)beta[1];
  } else {
    s.alpha = (T)alpha[0];
    s.beta = (T)beta[0];
  }
  s.beta_case = beta_case;
  return s;
}

template <class T>
static cudaError_t launch_add(const AddArgs &a, const double *alpha, const double *beta, int bcase,
                             cudaStream_t st) {
  const int64_t blocks = (a.total + 255) / 256;
  add_trace_kernel<T><<<(unsigned)(blocks < 148 * 32 ? blocks : 148 * 32), 256, 0, st>>>(
      a, add_scalars<T>(alpha, beta, bcase));
  return cudaGetLastError();
}

// Offsets reached by a view: [lo, hi] relative to its parent.
static int view_in_bounds(const qs_view *v, const char *name) {
  int64_t lo = v->offset, hi = v->offset;
  for (int d = 0; d < v->ndim; ++d) {
    if (v->size[d] == 0) return QS_OK;  // empty: reads nothing
    const int64_t span = (v->size[d] - 1) * v->strides[d];
    if (span < 0) lo += span; else hi += span;
  }
  if (lo < 0 || hi >= v->length) {
    std::ostringstream m;
    m << "BoundsError: " << name << " reaches offsets [" << lo << ", " << hi << "] of a parent of length "
      << v->length;
    return fail(QS_EBOUNDS, m.str());
  }
  return QS_OK;
}

}  // namespace qs

using namespace qs;

extern "C" int qs_tensoradd_trace(const qs_view *C, const double *alpha, const qs_view *A,
                                  const int64_t *indA, int32_t conjA, const double *beta,
                                  const int64_t *indC, void *stream) {
  int rc;
  if ((rc = validate_view(C, "C")) || (rc = validate_view(A, "A"))) return rc;
  if (!alpha || !beta) return fail(QS_EINVAL, "ArgumentError: alpha/beta is NULL");
  if ((A->ndim && !indA) || (C->ndim && !indC)) return fail(QS_EINVAL, "ArgumentError: label tuple is NULL");
  if (C->op == QS_OP_CONJ || C->op == QS_OP_ADJOINT)
    return fail(QS_EINVAL, "ArgumentError: the output C cannot be a conjugated view");
  if (!is_complex(C->eltype) && is_complex(A->eltype))
    return fail(QS_EINVAL, "ArgumentError: a complex A needs a complex C");
  const bool cx = is_complex(C->eltype) || is_complex(A->eltype);
  const bool dbl = is_double(C->eltype) || is_double(A->eltype);
  const int T = cx ? (dbl ? QS_C64 : QS_C32) : (dbl ? QS_F64 : QS_F32);
  if (!cx && (alpha[1] != 0.0 || beta[1] != 0.0))
    return fail(QS_EINVAL, "InexactError: a complex alpha/beta does not convert to the real compute type");
  if (C->ndim > kAddMaxRank) return fail(QS_EINVAL, "ArgumentError: C has more than 16 labels");
  AddArgs a{};
  // C labels: each once in C, once in A (same extent)
  for (int i = 0; i < C->ndim; ++i) {
    for (int j = 0; j < i; ++j)
      if (indC[j] == indC[i]) return fail(QS_EINVAL, "ArgumentError: a label appears twice in indC");
    int found = -1, count = 0;
    for (int j = 0; j < A->ndim; ++j)
      if (indA[j] == indC[i]) {
        found = j;
        ++count;
      }
    if (count != 1)
      return fail(QS_EINVAL, "ArgumentError: every label of indC must appear exactly once in indA");
    if (A->size[found] != C->size[i]) {
      std::ostringstream m;
      m << "DimensionMismatch: label " << indC[i] << " has length " << A->size[found] << " in A and "
        << C->size[i] << " in C";
      return fail(QS_EDIM, m.str());
    }
    a.csize[a.nc] = C->size[i];
    a.cstC[a.nc] = C->strides[i];
    a.cstA[a.nc] = A->strides[found];
    ++a.nc;
  }
  // the other labels of A: traced pairs
  for (int j = 0; j < A->ndim; ++j) {
    bool inC = false;
    for (int i = 0; i < C->ndim; ++i) inC |= indC[i] == indA[j];
    if (inC) continue;
    int first = -1, count = 0;
    for (int k = 0; k < A->ndim; ++k)
      if (indA[k] == indA[j]) {
        if (first < 0) first = k;
        ++count;
      }
    if (count != 2)
      return fail(QS_EINVAL, "ArgumentError: a label of indA that is not in indC must appear exactly twice "
                             "(a traced pair)");
    if (first != j) continue;  // the pair is added at its first occurrence
    int second = -1;
    for (int k = j + 1; k < A->ndim; ++k)
      if (indA[k] == indA[j]) second = k;
    if (A->size[j] != A->size[second])
      return fail(QS_EDIM, "DimensionMismatch: the two axes of a traced pair differ in length");
    if (a.nt >= kAddMaxRank) return fail(QS_EINVAL, "ArgumentError: more than 16 traced pairs");
    a.tsize[a.nt] = A->size[j];
    a.tstA[a.nt] = A->strides[j] + A->strides[second];
    ++a.nt;
  }
  a.total = 1;
  for (int d = 0; d < a.nc; ++d) a.total *= a.csize[d];
  a.tracelen = 1;
  for (int d = 0; d < a.nt; ++d) a.tracelen *= a.tsize[d];
  if (a.total == 0) return QS_OK;  // empty C: nothing to write
  const int acase = scalar_case(T, alpha), bcase = scalar_case(T, beta);
  a.read_a = (acase != 0 && a.tracelen > 0) ? 1 : 0;
  if ((rc = view_in_bounds(C, "C"))) return rc;
  if (a.read_a && (rc = view_in_bounds(A, "A"))) return rc;
  if (acase == 0 && bcase == 1) return QS_OK;  // C unchanged
  a.A = A->data;
  a.C = C->data;
  a.Abase = A->offset;
  a.Cbase = C->offset;
  a.TA = A->eltype;
  a.TC = C->eltype;
  a.conjA = ((conjA != 0) != (A->op == QS_OP_CONJ || A->op == QS_OP_ADJOINT)) ? 1 : 0;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  switch (T) {
    case QS_F32: e = launch_add<float>(a, alpha, beta, bcase, st); break;
    case QS_F64: e = launch_add<double>(a, alpha, beta, bcase, st); break;
    case QS_C32: e = launch_add<cplx<float>>(a, alpha, beta, bcase, st); break;
    default: e = launch_add<cplx<double>>(a, alpha, beta, bcase, st); break;
  }
  if (e != cudaSuccess) {
    std::ostringstream m;
    m << "CUDA error in the add/trace kernel launch: " << cudaGetErrorString(e);
    return fail(QS_ECUDA, m.str());
  }
  count_launches(1);
  return QS_OK;
}
