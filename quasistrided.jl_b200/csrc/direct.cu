// Gather kernels that read the operands in place through the plan's offset
// tables: the plain ("native") GEMM, C *= beta, the dot-product and the
// outer-product paths.
//
//   native GEMM   <- nest!/micro_tiles!/ScalarKernel (src/execution/nest.jl:7-191,
//                    src/microkernels/steps.jl:27-36): acc = muladd(a, b, acc)
//                    ascending in the plan's K order; complex in the planar
//                    kernel's fused order (steps.jl:121-167)
//   scale         <- scale_all_of_C! (src/execution/execute.jl:34-57)
//   dot           <- execute_path!(DotPath) (src/execution/dot.jl:13-76)
//   outer         <- execute_path!(OuterPath) (src/execution/outer.jl:10-69)
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "device_common.cuh"
#include "kernels.h"

namespace qs {

// ------------------------------------------------------------- scale ----

template <class T>
__global__ void scale_kernel(Operands op, Scalars<T> s, int mfast) {
  const int64_t mn = op.M * op.N, total = mn * op.P;
  for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < total;
       f += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = f / mn, e = f - b * mn;
    int64_t i, j;
    if (mfast) {
      i = e % op.M;
      j = e / op.M;
    } else {
      j = e % op.N;
      i = e / op.N;
    }
    int64_t idx = op.Cbase + op.offMC[i] + op.offNC[j];
    if (op.offBatch) idx += op.offBatch[2 * op.P + b];
    T v = s.beta_case == 0 ? tzero<T>() : cmul(load_c<T>(op.C, idx, op.TC), s.beta);
    store_c<T>(op.C, idx, op.TC, v);
  }
}

// -------------------------------------------------------- native GEMM ----
// Register-tiled gather GEMM: a CTA computes a BM x BN tile of C; its 256
// threads form an NTY x NTX grid, each owning TM x TN outputs (rows
// ty + NTY*i, columns tx + NTX*j).  A/B tiles are gathered through the
// offset tables (coalesced along whichever axis is unit-stride), converted
// to the compute type with conjugation on load, and double-buffered in
// shared memory.  The K loop runs over all of K, so beta is applied once.
// Tile shapes (DirectShape below) follow N: narrow-N problems get tall,
// narrow tiles instead of padding N to 64.

template <class T, int BM_, int BN_, int BK_, int TN_>
struct DirectCfg {
  static constexpr int BM = BM_, BN = BN_, BK = BK_, TN = TN_;
  static constexpr int kThreads = 256;
  static constexpr int NTX = BN / TN;
  static constexpr int NTY = kThreads / NTX;
  static constexpr int TM = BM / NTY;
  static constexpr int A_PER_THREAD = BM * BK / kThreads;
  static constexpr int B_PER_THREAD = (BN * BK + kThreads - 1) / kThreads;
  static_assert(NTX * NTY == kThreads && TM * NTY == BM && TN * NTX == BN, "tile shape");
  static_assert(A_PER_THREAD * kThreads == BM * BK, "A tile");
};

// The tile (bx, by) of one problem; the whole CTA calls it.
template <class T, class Cfg>
__device__ __forceinline__ void direct_gemm_tile(const Operands &op, const Scalars<T> &s,
                                                 int a_mfast, int b_nfast, int64_t bx, int64_t by) {
  constexpr int BM = Cfg::BM, BN = Cfg::BN, BK = Cfg::BK;
  constexpr int TM = Cfg::TM, TN = Cfg::TN, NTX = Cfg::NTX, NTY = Cfg::NTY;
  __shared__ T As[2][BK][BM];
  __shared__ T Bs[2][BK][BN];
  const int tid = threadIdx.x;
  const int tx = tid % NTX, ty = tid / NTX;
  const int64_t m0 = bx * BM, n0 = by * BN;

  T acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = tzero<T>();

  T ra[Cfg::A_PER_THREAD], rb[Cfg::B_PER_THREAD];
  auto a_coord = [&](int r, int &mm, int &kk) {
    int e = tid + r * Cfg::kThreads;
    if (a_mfast) { mm = e % BM; kk = e / BM; } else { kk = e % BK; mm = e / BK; }
  };
  auto b_coord = [&](int r, int &nn, int &kk) {
    int e = tid + r * Cfg::kThreads;
    if (b_nfast) { nn = e % BN; kk = e / BN; } else { kk = e % BK; nn = e / BK; }
    return e < BN * BK;
  };
  auto gather = [&](int64_t k0) {
#pragma unroll
    for (int r = 0; r < Cfg::A_PER_THREAD; ++r) {
      int mm, kk;
      a_coord(r, mm, kk);
      int64_t m = m0 + mm, k = k0 + kk;
      ra[r] = (m < op.M && k < op.K)
                  ? Loader<T>::load(op.A, op.Abase + op.offMA[m] + op.offKA[k], op.TA, op.conjA)
                  : tzero<T>();
    }
#pragma unroll
    for (int r = 0; r < Cfg::B_PER_THREAD; ++r) {
      int nn, kk;
      const bool in = b_coord(r, nn, kk);
      int64_t n = n0 + nn, k = k0 + kk;
      rb[r] = (in && n < op.N && k < op.K)
                  ? Loader<T>::load(op.B, op.Bbase + op.offNB[n] + op.offKB[k], op.TB, op.conjB)
                  : tzero<T>();
    }
  };
  auto stash = [&](int buf) {
#pragma unroll
    for (int r = 0; r < Cfg::A_PER_THREAD; ++r) {
      int mm, kk;
      a_coord(r, mm, kk);
      As[buf][kk][mm] = ra[r];
    }
#pragma unroll
    for (int r = 0; r < Cfg::B_PER_THREAD; ++r) {
      int nn, kk;
      if (b_coord(r, nn, kk)) Bs[buf][kk][nn] = rb[r];
    }
  };

  const int64_t nkb = (op.K + BK - 1) / BK;
  gather(0);
  stash(0);
  __syncthreads();
  for (int64_t kb = 0; kb < nkb; ++kb) {
    const int cur = kb & 1;
    if (kb + 1 < nkb) gather((kb + 1) * BK);
    const int64_t krem = op.K - kb * BK;
    const int kmax = krem < BK ? (int)krem : BK;
    for (int kk = 0; kk < kmax; ++kk) {
      T a[TM], b[TN];
#pragma unroll
      for (int i = 0; i < TM; ++i) a[i] = As[cur][kk][ty + NTY * i];
#pragma unroll
      for (int j = 0; j < TN; ++j) b[j] = Bs[cur][kk][tx + NTX * j];
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = cfma(a[i], b[j], acc[i][j]);
    }
    if (kb + 1 < nkb) stash(cur ^ 1);
    __syncthreads();
  }

#pragma unroll
  for (int i = 0; i < TM; ++i) {
    int64_t m = m0 + ty + NTY * i;
    if (m >= op.M) continue;
    int64_t cm = op.Cbase + op.offMC[m];
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      int64_t n = n0 + tx + NTX * j;
      if (n >= op.N) continue;
      int64_t idx = cm + op.offNC[n];
      T old = s.beta_case == 0 ? tzero<T>() : load_c<T>(op.C, idx, op.TC);
      store_c<T>(op.C, idx, op.TC, axpby(s, acc[i][j], old));
    }
  }
}

template <class T, class Cfg, bool BATCHED>
__global__ void __launch_bounds__(256) direct_gemm_kernel(Operands op, Scalars<T> s, int a_mfast,
                                                          int b_nfast) {
  if constexpr (!BATCHED) {
    direct_gemm_tile<T, Cfg>(op, s, a_mfast, b_nfast, blockIdx.x, blockIdx.y);
    return;
  }
  // Batch labels: this tile of every batch entry z, z + gridDim.z, ...
  for (int64_t b = blockIdx.z; b < op.P; b += gridDim.z) {
    direct_gemm_tile<T, Cfg>(batch_entry(op, b), s, a_mfast, b_nfast, blockIdx.x, blockIdx.y);
    __syncthreads();  // shared tiles are reused by the next entry
  }
}

// Tile shapes: 0 = 64 x 64 (N > 32), 1 = 128 x 32 (16 < N <= 32),
// 2 = 256 x 16 (N <= 16); complex compute types use 32 x 32 throughout.
template <class T, int SHAPE, bool CPLX = is_cplx<T>::value>
struct DirectShape;
template <class T>
struct DirectShape<T, 0, false> { using Cfg = DirectCfg<T, 64, 64, 16, 4>; };
template <class T>
struct DirectShape<T, 1, false> { using Cfg = DirectCfg<T, 128, 32, 16, 4>; };
template <class T>
struct DirectShape<T, 2, false> { using Cfg = DirectCfg<T, 256, 16, 8, 4>; };
template <class T>
struct DirectShape<T, 3, false> { using Cfg = DirectCfg<T, 32, 32, 16, 2>; };
template <class T, int SHAPE>
struct DirectShape<T, SHAPE, true> { using Cfg = DirectCfg<T, 32, 32, 16, 2>; };

// Plans: a small problem whose 64 x 64 grid would not fill the GPU takes
// 32 x 32 tiles (four times the CTAs).
int direct_shape_mn(int T, int64_t M, int64_t N) {
  int s = direct_shape(T, N);
  if (s == 0 && T != QS_C32 && T != QS_C64 && ((M + 63) / 64) * ((N + 63) / 64) < 148) s = 3;
  return s;
}

int direct_shape(int T, int64_t N) {
  if (T == QS_C32 || T == QS_C64) return 0;
  if (N <= 16) return 2;
  if (N <= 32) return 1;
  return 0;
}

// Grouped: CTA b runs tile b - block_start of the problem whose block range
// holds b (binary search over the NativeJob table); problems sorted by K
// descending so that the longest tiles start first.
template <class T, class Cfg>
__global__ void __launch_bounds__(256) direct_gemm_grouped_kernel(const NativeJob<T> *jobs, int njobs) {
  int lo = 0, hi = njobs - 1;
  const int b = blockIdx.x;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].block_start <= b) lo = mid;
    else hi = mid - 1;
  }
  const NativeJob<T> &j = jobs[lo];
  const int lb = b - j.block_start;
  const Operands op = j.op;
  const Scalars<T> s = j.s;
  direct_gemm_tile<T, Cfg>(op, s, j.a_mfast, j.b_nfast, lb % j.gx, lb / j.gx);
}

// ------------------------------------------------------------- skinny ----
// N <= 16 and K <= 64 (the read-B-in-place case: B is tiny, C and A are
// long): one thread per row of C, B and the K/N offset tables staged once per
// CTA in shared memory, K ascending with fma (the ScalarKernel order, as in
// the tiled kernel).  Bandwidth-bound: A is read once and C written once,
// with no tile padding along N.
constexpr int kSkinnyN = 16, kSkinnyK = 64;

int native_shape_for(int T, int TA, int TB, int64_t M, int64_t N, int64_t K, int native_tile, bool grouped) {
  // Problems the skinny kernel takes alone stay on the SIMT tiles in a
  // group too, so that a group's result equals its plans' own results.
  const bool dmma = dmma_eligible(T, TA, TB) && !(N <= kSkinnyN && K <= kSkinnyK);
  if (native_tile >= 1 && native_tile <= kSimtShapes) return is_complex(T) ? 0 : native_tile - 1;
  if (native_tile > kSimtShapes && native_tile <= kNativeShapes && dmma) return native_tile - 1;
  if (dmma) return kSimtShapes + (grouped ? dmma_shape_n(N) : dmma_shape_mn(M, N));
  return grouped ? direct_shape(T, N) : direct_shape_mn(T, M, N);
}

template <class T>
__device__ __forceinline__ void skinny_entry(const Operands &op, const Scalars<T> &s, T *Bs, int64_t *sKA,
                                             int64_t *sNC) {
  const int N = (int)op.N, K = (int)op.K;
  for (int e = threadIdx.x; e < K * N; e += blockDim.x) {
    const int k = e / N, j = e - k * N;
    Bs[k * kSkinnyN + j] = Loader<T>::load(op.B, op.Bbase + op.offNB[j] + op.offKB[k], op.TB, op.conjB);
  }
  for (int k = threadIdx.x; k < K; k += blockDim.x) sKA[k] = op.offKA[k];
  for (int j = threadIdx.x; j < N; j += blockDim.x) sNC[j] = op.offNC[j];
  __syncthreads();
  for (int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; m < op.M;
       m += (int64_t)gridDim.x * blockDim.x) {
    T acc[kSkinnyN];
#pragma unroll
    for (int j = 0; j < kSkinnyN; ++j) acc[j] = tzero<T>();
    const int64_t am = op.Abase + op.offMA[m];
    for (int k = 0; k < K; ++k) {
      const T a = Loader<T>::load(op.A, am + sKA[k], op.TA, op.conjA);
#pragma unroll
      for (int j = 0; j < kSkinnyN; ++j)
        if (j < N) acc[j] = cfma(a, Bs[k * kSkinnyN + j], acc[j]);
    }
    const int64_t cm = op.Cbase + op.offMC[m];
#pragma unroll
    for (int j = 0; j < kSkinnyN; ++j) {
      if (j >= N) break;
      const int64_t idx = cm + sNC[j];
      const T old = s.beta_case == 0 ? tzero<T>() : load_c<T>(op.C, idx, op.TC);
      store_c<T>(op.C, idx, op.TC, axpby(s, acc[j], old));
    }
  }
}

template <class T>
__global__ void __launch_bounds__(256) skinny_kernel(Operands op, Scalars<T> s) {
  __shared__ T Bs[kSkinnyK * kSkinnyN];
  __shared__ int64_t sKA[kSkinnyK], sNC[kSkinnyN];
  if (!op.offBatch) {
    skinny_entry<T>(op, s, Bs, sKA, sNC);
    return;
  }
  // Batch labels: entries y, y + gridDim.y, ... (B is staged per entry).
  for (int64_t b = blockIdx.y; b < op.P; b += gridDim.y) {
    skinny_entry<T>(batch_entry(op, b), s, Bs, sKA, sNC);
    __syncthreads();  // before the next entry overwrites the staged B
  }
}

// ---------------------------------------------------------------- dot ----
// out[q] = alpha * sum_k X[q,k] * v[k] + beta * C[q] for M == 1 or N == 1.
// kmode = 1: one warp per output, lanes stride K (K unit-stride in X);
// kmode = 0: one thread per output (Q unit-stride in X).

struct DotArgs {
  const void *X;  // matrix operand
  const void *V;  // vector operand
  int64_t Xbase, Vbase;
  int TX, TV;
  int conjX, conjV;
  const int64_t *offQX, *offKX, *offKV, *offQC;
  int x_is_a;  // X plays A (product a*b = X*v) or B (v*X)
  int64_t Q, K;
  void *C;
  int64_t Cbase;
  int TC;
};

template <class T>
__device__ __forceinline__ T dot_term(const DotArgs &d, int64_t q, int64_t k) {
  T x = Loader<T>::load(d.X, d.Xbase + d.offQX[q] + d.offKX[k], d.TX, d.conjX);
  T v = Loader<T>::load(d.V, d.Vbase + d.offKV[k], d.TV, d.conjV);
  return d.x_is_a ? cmul(x, v) : cmul(v, x);
}

template <class T>
__device__ __forceinline__ T shfl_down_t(T v, int o) {
  if constexpr (is_cplx<T>::value) {
    v.re = __shfl_down_sync(0xffffffffu, v.re, o);
    v.im = __shfl_down_sync(0xffffffffu, v.im, o);
    return v;
  } else {
    return __shfl_down_sync(0xffffffffu, v, o);
  }
}
template <class T>
__device__ __forceinline__ T tadd(T a, T b) {
  if constexpr (is_cplx<T>::value) {
    a.re += b.re;
    a.im += b.im;
    return a;
  } else {
    return a + b;
  }
}

template <class T>
__global__ void dot_kernel(DotArgs d, Scalars<T> s, int kmode) {
  if (kmode) {
    int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / 32;
    int lane = threadIdx.x & 31;
    int64_t nwarps = (int64_t)gridDim.x * blockDim.x / 32;
    for (int64_t q = warp; q < d.Q; q += nwarps) {
      T acc = tzero<T>();
      for (int64_t k = lane; k < d.K; k += 32) {
        T x = Loader<T>::load(d.X, d.Xbase + d.offQX[q] + d.offKX[k], d.TX, d.conjX);
        T v = Loader<T>::load(d.V, d.Vbase + d.offKV[k], d.TV, d.conjV);
        acc = d.x_is_a ? cfma(x, v, acc) : cfma(v, x, acc);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc = tadd(acc, shfl_down_t(acc, o));
      if (lane == 0) {
        int64_t idx = d.Cbase + d.offQC[q];
        T old = s.beta_case == 0 ? tzero<T>() : load_c<T>(d.C, idx, d.TC);
        store_c<T>(d.C, idx, d.TC, axpby(s, acc, old));
      }
    }
  } else {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < d.Q;
         q += (int64_t)gridDim.x * blockDim.x) {
      T acc = tzero<T>();
      const int64_t xq = d.Xbase + d.offQX[q];
      for (int64_t k = 0; k < d.K; ++k) {
        T x = Loader<T>::load(d.X, xq + d.offKX[k], d.TX, d.conjX);
        T v = Loader<T>::load(d.V, d.Vbase + d.offKV[k], d.TV, d.conjV);
        acc = d.x_is_a ? cfma(x, v, acc) : cfma(v, x, acc);
      }
      int64_t idx = d.Cbase + d.offQC[q];
      T old = s.beta_case == 0 ? tzero<T>() : load_c<T>(d.C, idx, d.TC);
      store_c<T>(d.C, idx, d.TC, axpby(s, acc, old));
    }
  }
}

// -------------------------------------------------------------- outer ----
// K == 1: C[i,j] = alpha * (a_i * b_j) + beta * C[i,j]; r = a*b then the
// store expression, term for term as the nest (src/execution/outer.jl:1-8).

template <class T>
__global__ void outer_kernel(Operands op, Scalars<T> s, int mfast) {
  int64_t total = op.M * op.N;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total;
       e += (int64_t)gridDim.x * blockDim.x) {
    int64_t i, j;
    if (mfast) { i = e % op.M; j = e / op.M; } else { j = e % op.N; i = e / op.N; }
    T a = Loader<T>::load(op.A, op.Abase + op.offMA[i] + op.offKA[0], op.TA, op.conjA);
    T b = Loader<T>::load(op.B, op.Bbase + op.offNB[j] + op.offKB[0], op.TB, op.conjB);
    T r = cmul(a, b);
    int64_t idx = op.Cbase + op.offMC[i] + op.offNC[j];
    T old = s.beta_case == 0 ? tzero<T>() : load_c<T>(op.C, idx, op.TC);
    store_c<T>(op.C, idx, op.TC, axpby(s, r, old));
  }
}

// ------------------------------------------------------------ launchers ---

static int grid_for(int64_t work, int threads) {
  int64_t g = (work + threads - 1) / threads;
  int64_t cap = 148 * 16;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

template <class T>
static cudaError_t launch_scale_t(const Operands &op, const double *alpha, const double *beta,
                                  int beta_case, int mfast, cudaStream_t st) {
  auto s = make_scalars<T>(alpha, beta, beta_case);
  scale_kernel<T><<<grid_for(op.M * op.N * op.P, 256), 256, 0, st>>>(op, s, mfast);
  return cudaGetLastError();
}

cudaError_t launch_scale(int T, const Operands &op, const double *beta, int beta_case, int mfast,
                         cudaStream_t st) {
  const double zero[2] = {0, 0};
  switch (T) {
    case QS_F32: return launch_scale_t<float>(op, zero, beta, beta_case, mfast, st);
    case QS_F64: return launch_scale_t<double>(op, zero, beta, beta_case, mfast, st);
    case QS_C32: return launch_scale_t<cplx<float>>(op, zero, beta, beta_case, mfast, st);
    default: return launch_scale_t<cplx<double>>(op, zero, beta, beta_case, mfast, st);
  }
}

template <class T, int SHAPE>
static cudaError_t launch_direct_s(const Operands &op, const Scalars<T> &s, int a_mfast, int b_nfast,
                                   cudaStream_t st) {
  using Cfg = typename DirectShape<T, SHAPE>::Cfg;
  dim3 grid((unsigned)((op.M + Cfg::BM - 1) / Cfg::BM), (unsigned)((op.N + Cfg::BN - 1) / Cfg::BN),
            (unsigned)(op.offBatch ? (op.P < 65535 ? op.P : 65535) : 1));
  if (op.offBatch)
    direct_gemm_kernel<T, Cfg, true><<<grid, 256, 0, st>>>(op, s, a_mfast, b_nfast);
  else
    direct_gemm_kernel<T, Cfg, false><<<grid, 256, 0, st>>>(op, s, a_mfast, b_nfast);
  return cudaGetLastError();
}

template <class T>
static cudaError_t launch_direct_t(int shape, const Operands &op, const double *alpha, const double *beta,
                                   int beta_case, int a_mfast, int b_nfast, cudaStream_t st) {
  auto s = make_scalars<T>(alpha, beta, beta_case);
  if (op.N <= kSkinnyN && op.K <= kSkinnyK) {
    const int64_t blocks = (op.M + 255) / 256;
    dim3 grid((unsigned)(blocks < 148 * 16 ? blocks : 148 * 16),
              (unsigned)(op.offBatch ? (op.P < 65535 ? op.P : 65535) : 1));
    skinny_kernel<T><<<grid, 256, 0, st>>>(op, s);
    return cudaGetLastError();
  }
  switch (shape) {
    case 1: return launch_direct_s<T, 1>(op, s, a_mfast, b_nfast, st);
    case 2: return launch_direct_s<T, 2>(op, s, a_mfast, b_nfast, st);
    case 3: return launch_direct_s<T, 3>(op, s, a_mfast, b_nfast, st);
    default: return launch_direct_s<T, 0>(op, s, a_mfast, b_nfast, st);
  }
}

cudaError_t launch_direct(int T, const Operands &op, const double *alpha, const double *beta,
                          int beta_case, int a_mfast, int b_nfast, int shape, cudaStream_t st) {
  if (shape >= kSimtShapes && dmma_eligible(T, op.TA, op.TB) && !(op.N <= kSkinnyN && op.K <= kSkinnyK))
    return launch_dmma(op, alpha, beta, beta_case, a_mfast, b_nfast, shape - kSimtShapes, st);
  if (shape >= kSimtShapes) shape = 0;
  switch (T) {
    case QS_F32: return launch_direct_t<float>(shape, op, alpha, beta, beta_case, a_mfast, b_nfast, st);
    case QS_F64: return launch_direct_t<double>(shape, op, alpha, beta, beta_case, a_mfast, b_nfast, st);
    case QS_C32: return launch_direct_t<cplx<float>>(0, op, alpha, beta, beta_case, a_mfast, b_nfast, st);
    default: return launch_direct_t<cplx<double>>(0, op, alpha, beta, beta_case, a_mfast, b_nfast, st);
  }
}

template <class T>
static cudaError_t launch_dot_t(const DotArgs &d, const double *alpha, const double *beta,
                                int beta_case, int kmode, cudaStream_t st) {
  auto s = make_scalars<T>(alpha, beta, beta_case);
  int threads = 256;
  int64_t work = kmode ? d.Q * 32 : d.Q;
  dot_kernel<T><<<grid_for(work, threads), threads, 0, st>>>(d, s, kmode);
  return cudaGetLastError();
}

cudaError_t launch_dot(int T, const Operands &op, const double *alpha, const double *beta,
                       int beta_case, cudaStream_t st) {
  DotArgs d;
  if (op.N == 1) {  // X = A (Q = M), v = B
    d.X = op.A; d.V = op.B; d.Xbase = op.Abase; d.Vbase = op.Bbase + 0;
    d.TX = op.TA; d.TV = op.TB; d.conjX = op.conjA; d.conjV = op.conjB;
    d.offQX = op.offMA; d.offKX = op.offKA; d.offKV = op.offKB; d.offQC = op.offMC;
    d.x_is_a = 1; d.Q = op.M;
    d.Vbase = op.Bbase;  // the single N coordinate has offset 0
  } else {          // M == 1: X = B (Q = N), v = A
    d.X = op.B; d.V = op.A; d.Xbase = op.Bbase; d.Vbase = op.Abase;
    d.TX = op.TB; d.TV = op.TA; d.conjX = op.conjB; d.conjV = op.conjA;
    d.offQX = op.offNB; d.offKX = op.offKB; d.offKV = op.offKA; d.offQC = op.offNC;
    d.x_is_a = 0; d.Q = op.N;
  }
  d.K = op.K;
  d.C = op.C;
  d.Cbase = op.Cbase;
  d.TC = op.TC;
  int kmode = 1;  // default: warp per output
  switch (T) {
    case QS_F32: return launch_dot_t<float>(d, alpha, beta, beta_case, kmode, st);
    case QS_F64: return launch_dot_t<double>(d, alpha, beta, beta_case, kmode, st);
    case QS_C32: return launch_dot_t<cplx<float>>(d, alpha, beta, beta_case, kmode, st);
    default: return launch_dot_t<cplx<double>>(d, alpha, beta, beta_case, kmode, st);
  }
}

template <class T>
static cudaError_t launch_outer_t(const Operands &op, const double *alpha, const double *beta,
                                  int beta_case, int mfast, cudaStream_t st) {
  auto s = make_scalars<T>(alpha, beta, beta_case);
  outer_kernel<T><<<grid_for(op.M * op.N, 256), 256, 0, st>>>(op, s, mfast);
  return cudaGetLastError();
}

cudaError_t launch_outer(int T, const Operands &op, const double *alpha, const double *beta,
                         int beta_case, int mfast, cudaStream_t st) {
  switch (T) {
    case QS_F32: return launch_outer_t<float>(op, alpha, beta, beta_case, mfast, st);
    case QS_F64: return launch_outer_t<double>(op, alpha, beta, beta_case, mfast, st);
    case QS_C32: return launch_outer_t<cplx<float>>(op, alpha, beta, beta_case, mfast, st);
    default: return launch_outer_t<cplx<double>>(op, alpha, beta, beta_case, mfast, st);
  }
}

template <class T>
static int native_group_build_t(NativeGroup &g, const Operands *ops, const double *alpha,
                                const double *beta, const int *bcase) {
  const int n = (int)g.plans.size();
  std::vector<NativeJob<T>> jobs(n);
  int64_t blocks = 0;
  for (int i = 0; i < n; ++i) {
    const int k = g.idx[i];
    NativeJob<T> &j = jobs[i];
    j.op = ops[i];
    j.s = make_scalars<T>(alpha + 2 * k, beta + 2 * k, bcase[k]);
    j.a_mfast = g.plans[i]->a_mfast;
    j.b_nfast = g.plans[i]->b_nfast;
    int bm = 64, bn = 64;
    if (g.shape >= kSimtShapes) dmma_tile_dims(g.shape - kSimtShapes, &bm, &bn);
    else if (is_complex(g.T)) bm = bn = 32;
    else if (g.shape == 1) bm = 128, bn = 32;
    else if (g.shape == 2) bm = 256, bn = 16;
    else if (g.shape == 3) bm = 32, bn = 32;
    const int64_t gx = (j.op.M + bm - 1) / bm, gy = (j.op.N + bn - 1) / bn;
    if (gx > INT32_MAX || blocks + gx * gy > INT32_MAX) return fail(QS_EINVAL, "ArgumentError: grouped launch too large");
    j.gx = (int)gx;
    j.block_start = (int)blocks;
    blocks += gx * gy;
  }
  g.blocks = (int)blocks;
  g.image.resize(n * sizeof(NativeJob<T>));
  std::memcpy(g.image.data(), jobs.data(), g.image.size());
  return QS_OK;
}

int native_group_build(NativeGroup &g, const Operands *ops, const double *alpha, const double *beta,
                       const int *bcase) {
  switch (g.T) {
    case QS_F32: return native_group_build_t<float>(g, ops, alpha, beta, bcase);
    case QS_F64: return native_group_build_t<double>(g, ops, alpha, beta, bcase);
    case QS_C32: return native_group_build_t<cplx<float>>(g, ops, alpha, beta, bcase);
    default: return native_group_build_t<cplx<double>>(g, ops, alpha, beta, bcase);
  }
}

template <class T, int SHAPE>
static void native_group_launch_s(const NativeGroup &g, cudaStream_t st) {
  using Cfg = typename DirectShape<T, SHAPE>::Cfg;
  direct_gemm_grouped_kernel<T, Cfg><<<g.blocks, 256, 0, st>>>((const NativeJob<T> *)g.dev, (int)g.plans.size());
}

template <class T>
static cudaError_t native_group_launch_t(const NativeGroup &g, cudaStream_t st) {
  switch (g.shape) {
    case 1: native_group_launch_s<T, 1>(g, st); break;
    case 2: native_group_launch_s<T, 2>(g, st); break;
    case 3: native_group_launch_s<T, 3>(g, st); break;
    default: native_group_launch_s<T, 0>(g, st); break;
  }
  return cudaGetLastError();
}

cudaError_t native_group_launch(const NativeGroup &g, cudaStream_t st) {
  if (g.plans.empty()) return cudaSuccess;
  if (g.shape >= kSimtShapes)
    return dmma_group_launch(g.shape - kSimtShapes, g.dev, (int)g.plans.size(), g.blocks, st);
  switch (g.T) {
    case QS_F32: return native_group_launch_t<float>(g, st);
    case QS_F64: return native_group_launch_t<double>(g, st);
    case QS_C32: return native_group_launch_t<cplx<float>>(g, st);
    default: return native_group_launch_t<cplx<double>>(g, st);
  }
}

}  // namespace qs
