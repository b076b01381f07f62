// The plain native-FP64 GEMM on the FP64 tensor cores (DMMA, mma.sync
// m16n8k8 .f64), for real Float64 operands: the device counterpart of
// nest!/micro_tiles! with SIMDKernel's Float64 FMA tile
// (src/execution/nest.jl:7-122, src/microkernels/steps.jl:73-106).
//
// A CTA computes a BM x BN tile of C over all of K (beta applied once, as
// nest.jl:83 applies it on the first K block only).  The operands are never
// packed: every K tile of A and B is gathered straight from the caller's
// strided storage through the plan's offset tables, element by element with
// 8-byte cp.async (zero-filled outside M/N/K), into a STAGES-deep ring of
// shared-memory tiles.  The gather walks whichever axis is unit-stride in
// global memory (rows or K), so the loads coalesce for either layout.
//
// Shared-memory tile: one row of 16 doubles (one K tile) per M (or N)
// index.  Within each 8-wide K block, K index kk sits at position
// 2*(kk & 3) + (kk >> 2): the two values a thread's fragment takes from a
// row (K = tig and tig + 4) are adjacent, so one 16-byte load fetches them.
// The 16-byte chunks of a row are XOR-swizzled by the row's low three bits
// (odd rows flip chunk bit 2, rows 2q and 2q+1 flip bits 0-1 by q), which
// makes every fragment load conflict-free and spreads the row-wise cp.async
// writes over eight chunk positions.
//
// Arithmetic: each DMMA adds eight products to the FP64 accumulator; the
// K order is the plan's, ascending.  The epilogue is axpby with the
// Zero/One/beta cases and one rounding to eltype(C), as in the gather GEMM.
#include <cuda_runtime.h>

#include <atomic>
#include <climits>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "device_common.cuh"
#include "kernels.h"
#include "ptx.cuh"

namespace qs {

template <int BM_, int BN_, int WGM_, int WGN_, int STAGES_>
struct DmmaCfg {
  static constexpr int BM = BM_, BN = BN_, WGM = WGM_, WGN = WGN_, STAGES = STAGES_;
  static constexpr int BK = 16;
  static constexpr int kWarps = WGM * WGN, kThreads = 32 * kWarps;
  static constexpr int WM = BM / WGM, WN = BN / WGN;  // warp tile
  static constexpr int MI = WM / 16, NJ = WN / 8;     // mma tiles per warp
  static constexpr int A_PER = BM * BK / kThreads, B_PER = BN * BK / kThreads;
  static constexpr int STAGE_DOUBLES = (BM + BN) * BK;
  static constexpr size_t kSmem = (size_t)STAGES * STAGE_DOUBLES * 8 + (size_t)(BM + BN) * 8;
  static_assert(MI * 16 * WGM == BM && NJ * 8 * WGN == BN, "warp tiling");
  static_assert(A_PER * kThreads == BM * BK && B_PER * kThreads == BN * BK, "gather split");
};

// Position (in doubles) of element (row r, K index k < 16) in a tile.
__device__ __forceinline__ int dmma_swz(int r) { return ((r & 1) << 2) | ((r >> 1) & 3); }
__device__ __forceinline__ int dmma_pos(int r, int k) {
  const int kk = k & 7;
  const int chunk = ((k >> 3) << 2) | (kk & 3);
  return r * 16 + 2 * (chunk ^ dmma_swz(r)) + (kk >> 2);
}


__device__ __forceinline__ void dmma_16x8x8(double (&c)[4], const double (&a)[4], const double (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

// Gathers K tile [k0, k0 + 16) of one operand (rows R of the CTA tile) into
// `tile`.  rowoff[r] is the row's offset (INT64_MIN outside the operand);
// rfast: rows are the operand's unit-stride axis.
template <int R, int PER, int THREADS>
__device__ __forceinline__ void dmma_gather(const double *X, const int64_t *rowoff, const int64_t *offK,
                                            int64_t k0, int64_t K, int rfast, uint32_t tile) {
  static_assert(THREADS % R == 0 ? (THREADS / R) * PER == 16 : false, "row-fast gather covers the K tile");
  static_assert((THREADS / 16) * PER == R, "K-fast gather covers the rows");
  const int tid = threadIdx.x;
  if (rfast) {
    // consecutive threads take consecutive rows; K steps by THREADS / R
    constexpr int KSTEP = THREADS / R;
    const int r = tid % R, kb = tid / R;
    const int64_t ro = rowoff[r];
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      const int k = kb + KSTEP * j;
      const int64_t kg = k0 + k;
      const bool ok = ro != INT64_MIN && kg < K;
      const double *src = ok ? X + ro + __ldg(offK + kg) : X;
      cp_async8(tile + 8u * (uint32_t)dmma_pos(r, k), src, ok ? 8 : 0);
    }
  } else {
    // sixteen consecutive threads take one row's K tile
    constexpr int RSTEP = THREADS / 16;
    const int k = tid & 15, rb = tid >> 4;
    const int64_t kg = k0 + k;
    const int64_t ko = kg < K ? __ldg(offK + kg) : INT64_MIN;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      const int r = rb + RSTEP * j;
      const int64_t ro = rowoff[r];
      const bool ok = ro != INT64_MIN && ko != INT64_MIN;
      const double *src = ok ? X + ro + ko : X;
      cp_async8(tile + 8u * (uint32_t)dmma_pos(r, k), src, ok ? 8 : 0);
    }
  }
}

// The tile (tm, tn) of one problem; the whole CTA calls it.  `smem` is the
// dynamic shared memory (Cfg::kSmem bytes).
template <class Cfg>
__device__ __forceinline__ void dmma_gemm_tile(const Operands &op, const Scalars<double> &s, int a_mfast,
                                               int b_nfast, int64_t tm, int64_t tn, double *smem) {
  constexpr int BM = Cfg::BM, BN = Cfg::BN, STAGES = Cfg::STAGES, MI = Cfg::MI, NJ = Cfg::NJ;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, tig = lane & 3;
  const int wm = warp % Cfg::WGM, wn = warp / Cfg::WGM;
  const int64_t m0 = tm * BM, n0 = tn * BN;

  int64_t *rowA = reinterpret_cast<int64_t *>(smem + (size_t)STAGES * Cfg::STAGE_DOUBLES);
  int64_t *rowB = rowA + BM;
  for (int r = tid; r < BM; r += Cfg::kThreads) {
    const int64_t m = m0 + r;
    rowA[r] = m < op.M ? op.Abase + __ldg(op.offMA + m) : INT64_MIN;
  }
  for (int r = tid; r < BN; r += Cfg::kThreads) {
    const int64_t n = n0 + r;
    rowB[r] = n < op.N ? op.Bbase + __ldg(op.offNB + n) : INT64_MIN;
  }
  __syncthreads();

  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(smem);
  auto stage_a = [&](int st) { return sbase + 8u * (uint32_t)(st * Cfg::STAGE_DOUBLES); };
  auto stage_b = [&](int st) { return sbase + 8u * (uint32_t)(st * Cfg::STAGE_DOUBLES + BM * 16); };
  const double *Ap = static_cast<const double *>(op.A);
  const double *Bp = static_cast<const double *>(op.B);
  const int64_t nkt = (op.K + 15) / 16;
  auto load = [&](int64_t kt) {
    const int st = (int)(kt % STAGES);
    dmma_gather<BM, Cfg::A_PER, Cfg::kThreads>(Ap, rowA, op.offKA, kt * 16, op.K, a_mfast, stage_a(st));
    dmma_gather<BN, Cfg::B_PER, Cfg::kThreads>(Bp, rowB, op.offKB, kt * 16, op.K, b_nfast, stage_b(st));
  };

  double acc[MI][NJ][4];
#pragma unroll
  for (int i = 0; i < MI; ++i)
#pragma unroll
    for (int j = 0; j < NJ; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.0;

#pragma unroll
  for (int st = 0; st < STAGES - 1; ++st) {
    if (st < nkt) load(st);
    cp_async_commit();
  }
  for (int64_t kt = 0; kt < nkt; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();  // tile kt landed for every thread; stage (kt - 1) % STAGES is free
    if (kt + STAGES - 1 < nkt) load(kt + STAGES - 1);
    cp_async_commit();
    const int st = (int)(kt % STAGES);
    const double *As = smem + (size_t)st * Cfg::STAGE_DOUBLES;
    const double *Bs = As + BM * 16;
#pragma unroll
    for (int kb = 0; kb < 2; ++kb) {
      double bf[NJ][2];
#pragma unroll
      for (int j = 0; j < NJ; ++j) {
        const int r = wn * Cfg::WN + 8 * j + g;
        const double2 v = *reinterpret_cast<const double2 *>(Bs + r * 16 + 2 * ((kb * 4 + tig) ^ dmma_swz(r)));
        bf[j][0] = v.x;
        bf[j][1] = v.y;
      }
#pragma unroll
      for (int i = 0; i < MI; ++i) {
        const int r = wm * Cfg::WM + 16 * i + g;
        const double2 lo = *reinterpret_cast<const double2 *>(As + r * 16 + 2 * ((kb * 4 + tig) ^ dmma_swz(r)));
        const double2 hi =
            *reinterpret_cast<const double2 *>(As + (r + 8) * 16 + 2 * ((kb * 4 + tig) ^ dmma_swz(r + 8)));
        const double af[4] = {lo.x, hi.x, lo.y, hi.y};
#pragma unroll
        for (int j = 0; j < NJ; ++j) dmma_16x8x8(acc[i][j], af, bf[j]);
      }
    }
  }
  cp_async_wait<0>();

  // Epilogue: rows g, g + 8 of each m16 tile, columns 2 tig, 2 tig + 1 of
  // each n8 tile.
  int64_t cn[NJ][2];
#pragma unroll
  for (int j = 0; j < NJ; ++j)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int64_t n = n0 + wn * Cfg::WN + 8 * j + 2 * tig + h;
      cn[j][h] = n < op.N ? __ldg(op.offNC + n) : INT64_MIN;
    }
#pragma unroll
  for (int i = 0; i < MI; ++i)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int64_t m = m0 + wm * Cfg::WM + 16 * i + g + 8 * h;
      if (m >= op.M) continue;
      const int64_t cm = op.Cbase + __ldg(op.offMC + m);
#pragma unroll
      for (int j = 0; j < NJ; ++j)
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          if (cn[j][c] == INT64_MIN) continue;
          const int64_t idx = cm + cn[j][c];
          const double old = s.beta_case == 0 ? 0.0 : load_c<double>(op.C, idx, op.TC);
          store_c<double>(op.C, idx, op.TC, axpby(s, acc[i][j][2 * h + c], old));
        }
    }
}

// Tiles in bands of `kBand` M tiles, N tiles within a band: a wave of CTAs
// shares few A and B panels in L2.
__device__ __forceinline__ void dmma_band(int64_t b, int64_t gm, int64_t gn, int64_t kBand, int64_t &tm,
                                          int64_t &tn) {
  const int64_t per = kBand * gn;
  const int64_t band = b / per, r = b - band * per;
  const int64_t rows = (band + 1) * kBand <= gm ? kBand : gm - band * kBand;
  tm = band * kBand + r % rows;
  tn = r / rows;
}

template <class Cfg, bool BATCHED>
__global__ void __launch_bounds__(Cfg::kThreads, 1)
    dmma_gemm_kernel(const __grid_constant__ Operands op, const Scalars<double> s, int a_mfast, int b_nfast,
                     int band) {
  extern __shared__ __align__(128) double dsm[];
  const int64_t gm = (op.M + Cfg::BM - 1) / Cfg::BM, gn = (op.N + Cfg::BN - 1) / Cfg::BN;
  int64_t tm, tn;
  dmma_band(blockIdx.x, gm, gn, band, tm, tn);
  if constexpr (!BATCHED) {
    dmma_gemm_tile<Cfg>(op, s, a_mfast, b_nfast, tm, tn, dsm);
  } else {
    for (int64_t b = blockIdx.z; b < op.P; b += gridDim.z) {
      dmma_gemm_tile<Cfg>(batch_entry(op, b), s, a_mfast, b_nfast, tm, tn, dsm);
      __syncthreads();  // the next entry reuses the shared tiles
    }
  }
}

// Grouped: CTA b runs tile b - block_start of the problem whose block range
// holds b (binary search over the K-descending job table).
template <class Cfg>
__global__ void __launch_bounds__(Cfg::kThreads, 1) dmma_gemm_grouped_kernel(const NativeJob<double> *jobs,
                                                                             int njobs) {
  extern __shared__ __align__(128) double dsm[];
  int lo = 0, hi = njobs - 1;
  const int b = blockIdx.x;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].block_start <= b) lo = mid;
    else hi = mid - 1;
  }
  const NativeJob<double> &j = jobs[lo];
  const int lb = b - j.block_start;
  dmma_gemm_tile<Cfg>(j.op, j.s, j.a_mfast, j.b_nfast, lb % j.gx, lb / j.gx, dsm);
}

// Shapes: 0 = 128 x 128 (8 warps of 64 x 32), 1 = 128 x 64 (8 warps of
// 32 x 32), 2 = 64 x 64 (4 warps of 32 x 32), 3 = 128 x 32 (8 warps of
// 16 x 32), 4 = 256 x 16 (8 warps of 32 x 16).
template <int SHAPE>
struct DmmaShape;
template <>
struct DmmaShape<0> { using Cfg = DmmaCfg<128, 128, 2, 4, 4>; };
template <>
struct DmmaShape<1> { using Cfg = DmmaCfg<128, 64, 4, 2, 4>; };
template <>
struct DmmaShape<2> { using Cfg = DmmaCfg<64, 64, 2, 2, 4>; };
template <>
struct DmmaShape<3> { using Cfg = DmmaCfg<128, 32, 8, 1, 4>; };
template <>
struct DmmaShape<4> { using Cfg = DmmaCfg<256, 16, 8, 1, 3>; };  // 104 KB: two CTAs per SM
template <>
struct DmmaShape<5> { using Cfg = DmmaCfg<128, 128, 4, 4, 4>; };

void dmma_tile_dims(int shape, int *bm, int *bn) {
  switch (shape) {
    case 1: *bm = 128; *bn = 64; break;
    case 2: *bm = 64; *bn = 64; break;
    case 3: *bm = 128; *bn = 32; break;
    case 4: *bm = 256; *bn = 16; break;
    case 5: *bm = 128; *bn = 128; break;
    default: *bm = 128; *bn = 128; break;
  }
}

// M tiles per raster band.  Bands of 8 to 64 M tiles measured within 5 % of
// each other on the 4096 x 4096 x 2304 permuted contraction, and
// evict-first C traffic made no difference.
constexpr int kDmmaBandM = 32;
static int dmma_band_m() { return kDmmaBandM; }

bool dmma_eligible(int T, int TA, int TB) { return T == QS_F64 && TA == QS_F64 && TB == QS_F64; }

// By N: 64 x 64 tiles (4 warps, three CTAs per SM) for N > 32 -- on the
// 4096 x 4096 x 2304 permuted contraction they beat 128 x 128 with 8 warps
// (one CTA per SM) 22.8 to 20.0 TFLOP/s, and 128 x 128 with 16 warps (21.3):
// independent CTAs hide each other's pipeline stalls; narrow N takes tall,
// narrow tiles instead of padding N.
int dmma_shape_n(int64_t N) {
  if (N <= 16) return 4;
  if (N <= 32) return 3;
  return 2;
}

int dmma_shape_mn(int64_t M, int64_t N) {
  (void)M;
  return dmma_shape_n(N);
}

// The dynamic shared-memory opt-in of one kernel instance, set on the
// first launch on each device (a per-launch driver call costs microseconds
// on the one-shot contract path).  KERNEL makes the flag one per kernel:
// instances of one signature share a function-pointer type.
template <class Cfg, auto KERNEL>
static cudaError_t dmma_smem_attr() {
  static std::atomic<uint64_t> done{0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 63;
  const uint64_t bit = 1ull << dev;
  if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
  const cudaError_t e =
      cudaFuncSetAttribute(KERNEL, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Cfg::kSmem);
  if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_release);
  return e;
}

template <int SHAPE>
static cudaError_t launch_dmma_s(const Operands &op, const Scalars<double> &s, int a_mfast, int b_nfast,
                                 cudaStream_t st) {
  using Cfg = typename DmmaShape<SHAPE>::Cfg;
  const int64_t gm = (op.M + Cfg::BM - 1) / Cfg::BM, gn = (op.N + Cfg::BN - 1) / Cfg::BN;
  if (gm * gn > INT_MAX) return cudaErrorInvalidConfiguration;
  dim3 grid((unsigned)(gm * gn), 1, (unsigned)(op.offBatch ? (op.P < 65535 ? op.P : 65535) : 1));
  cudaError_t e;
  if (op.offBatch) {
    if ((e = dmma_smem_attr<Cfg, dmma_gemm_kernel<Cfg, true>>()) != cudaSuccess) return e;
    dmma_gemm_kernel<Cfg, true><<<grid, Cfg::kThreads, Cfg::kSmem, st>>>(op, s, a_mfast, b_nfast, dmma_band_m());
  } else {
    if ((e = dmma_smem_attr<Cfg, dmma_gemm_kernel<Cfg, false>>()) != cudaSuccess) return e;
    dmma_gemm_kernel<Cfg, false><<<grid, Cfg::kThreads, Cfg::kSmem, st>>>(op, s, a_mfast, b_nfast, dmma_band_m());
  }
  return cudaGetLastError();
}

cudaError_t launch_dmma(const Operands &op, const double *alpha, const double *beta, int beta_case,
                        int a_mfast, int b_nfast, int shape, cudaStream_t st) {
  const Scalars<double> s = make_scalars<double>(alpha, beta, beta_case);
  switch (shape) {
    case 1: return launch_dmma_s<1>(op, s, a_mfast, b_nfast, st);
    case 2: return launch_dmma_s<2>(op, s, a_mfast, b_nfast, st);
    case 3: return launch_dmma_s<3>(op, s, a_mfast, b_nfast, st);
    case 4: return launch_dmma_s<4>(op, s, a_mfast, b_nfast, st);
    case 5: return launch_dmma_s<5>(op, s, a_mfast, b_nfast, st);
    default: return launch_dmma_s<0>(op, s, a_mfast, b_nfast, st);
  }
}

template <int SHAPE>
static cudaError_t dmma_group_launch_s(const void *jobs, int njobs, int blocks, cudaStream_t st) {
  using Cfg = typename DmmaShape<SHAPE>::Cfg;
  cudaError_t e = dmma_smem_attr<Cfg, dmma_gemm_grouped_kernel<Cfg>>();
  if (e != cudaSuccess) return e;
  dmma_gemm_grouped_kernel<Cfg>
      <<<blocks, Cfg::kThreads, Cfg::kSmem, st>>>(static_cast<const NativeJob<double> *>(jobs), njobs);
  return cudaGetLastError();
}

cudaError_t dmma_group_launch(int shape, const void *jobs, int njobs, int blocks, cudaStream_t st) {
  switch (shape) {
    case 1: return dmma_group_launch_s<1>(jobs, njobs, blocks, st);
    case 2: return dmma_group_launch_s<2>(jobs, njobs, blocks, st);
    case 3: return dmma_group_launch_s<3>(jobs, njobs, blocks, st);
    case 4: return dmma_group_launch_s<4>(jobs, njobs, blocks, st);
    case 5: return dmma_group_launch_s<5>(jobs, njobs, blocks, st);
    default: return dmma_group_launch_s<0>(jobs, njobs, blocks, st);
  }
}

}  // namespace qs
