// Tensor-core paths of the nest (execute_path!(NestPath), src/execution/nest.jl:7-191):
//
//  * Float64 as an Ozaki-style split: every row of A and every column of B is
//    scaled by a power of two (its max-magnitude exponent), cut into s signed
//    balanced base-256 digits (int8), and the slice products are
//    computed exactly on the integer tensor cores (tcgen05.mma kind::i8,
//    INT32 accumulation in TMEM).
//    Products of equal weight (p + q = t) share one INT32 accumulator; each
//    diagonal is added into an FP64 running sum kept in TMEM, and the final
//    alpha/beta epilogue rescales and rounds once to eltype(C).
//  * Float32 as split-BF16 x3: hi = bf16(x), lo = bf16(x - hi); the products
//    hi*hi + hi*lo + lo*hi accumulate in FP32 in TMEM (kind::f16).
//
// Packing (src/packing/pack.jl:43-99) becomes a device pass that gathers each
// operand through its offset tables, converts it to the compute type with
// conjugation on load, and writes K-major panels in the exact byte image of
// the 128-byte-swizzled shared-memory tiles the MMA reads, so the GEMM moves
// whole tiles with single bulk copies.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <sstream>
#include <utility>
#include <vector>

#include "kernels.h"
#include "ptx.cuh"
#include "tc.h"

namespace qs {

constexpr int kTileM = 128;     // UMMA M
constexpr int kKBytes = 128;    // bytes of K per panel tile (one swizzle row)
constexpr int kNonFinite = INT_MIN;

// x * 2^e.  When 2^e is a normal double the product is one multiplication
// by an exactly built power of two (exact, or rounded once if the result is
// subnormal), which is ldexp's result; other e take ldexp.
__device__ __noinline__ double scale2_wide(double x, int e) { return ldexp(x, e); }
__device__ __forceinline__ double scale2(double x, int e) {
  if (e >= -1022 && e <= 1023) return x * __longlong_as_double((long long)(e + 1023) << 52);
  return scale2_wide(x, e);
}

// ------------------------------------------------------------- packing ---

struct PackArgs {
  const void *X;
  int64_t Xbase;
  int TX, conj;
  const int64_t *offR, *offK;  // row (M or N) and K offset tables of X
  int64_t rows, K;             // logical extents
  int64_t rows_pad;            // padded to the panel tile height
  int tile_rows;               // 128 or 256
  int kblocks;                 // K bytes / 128 per padded row
  int rfast;                   // rows are X's unit-stride axis
  uint8_t *panel;
  int64_t plane;  // bytes per slice plane
  int nslices;
  int32_t *exp_out;
  int32_t *flag_list, *flag_count;
  // Complex operands as real matrices: 0 = real; 1 = "1e" (row 2i =
  // [re, -im], row 2i+1 = [im, re] along K pairs; rows and K are doubled);
  // 2 = "1r" (K pair = [re; im]; K doubled).  The 1m layout packs A as 1e
  // and B as 1r; the planar layout A as 1r and B as 1e, so that a real row
  // of C holds (re, im) of each complex element in adjacent columns.
  // `rows`/`K` above are the real (virtual) extents; offR/offK index the
  // complex elements.
  int cmode;
  // Ozaki pass 1 -> pass 2: each padded row's max |x| bit pattern (zeroed
  // before every pack), or nullptr.
  unsigned long long *rowmax;
  // The order in which the pack visits rows (rows_pad entries: tile row i
  // is virtual row rperm[i]), or nullptr for 0, 1, 2, ...  A real operand
  // whose unit-stride axis is a later label of its row group gets the order
  // with that label fastest, so a warp's 32 rows are adjacent in memory.
  const int32_t *rperm;
};

// Virtual row of the pack's row position i.
__device__ __forceinline__ int64_t pack_row(const PackArgs &a, int64_t i) {
  return a.rperm ? (int64_t)__ldg(a.rperm + i) : i;
}

// Element (r, k) of the real (virtual) matrix the panels hold.
template <class T>
__device__ __forceinline__ T virtual_elem(const PackArgs &a, int64_t r, int64_t k) {
  if (a.cmode == 0) return Loader<T>::load(a.X, a.Xbase + a.offR[r] + a.offK[k], a.TX, a.conj);
  using C = cplx<T>;
  if (a.cmode == 1) {
    const C z = Loader<C>::load(a.X, a.Xbase + a.offR[r >> 1] + a.offK[k >> 1], a.TX, a.conj);
    const int rp = (int)(r & 1), kp = (int)(k & 1);
    return rp == kp ? z.re : (rp ? z.im : -z.im);
  }
  const C z = Loader<C>::load(a.X, a.Xbase + a.offR[r] + a.offK[k >> 1], a.TX, a.conj);
  return (k & 1) ? z.im : z.re;
}

__device__ __forceinline__ int64_t panel_tile_base(const PackArgs &a, int64_t row, int64_t kbyte) {
  int64_t rt = row / a.tile_rows, r = row % a.tile_rows;
  int64_t kb = kbyte >> 7;
  return ((rt * a.kblocks + kb) * a.tile_rows) * kKBytes + sw128_offset((uint32_t)r, (uint32_t)(kbyte & 127));
}

// A tile of 32 rows x KT K values of X, converted to the compute type, into
// smem, coalesced along whichever of rows / K is X's unit-stride axis.
// Column skew of the pack tiles: element k of a row sits at column
// tcol(k), which rotates each group of W = KT/8 columns by its group index.
// The readers take W consecutive columns per thread, eight threads per row;
// without the skew those eight threads hit one bank.
template <int KT>
__device__ __forceinline__ int tcol(int k) {
  constexpr int W = KT / 8;
  return (k & ~(W - 1)) | ((k + k / W) & (W - 1));
}

// Real operands stored as S: each thread keeps the offset of its fixed row
// (or K index) in a register and issues all of its loads independently.
template <class T, class S, int KT>
__device__ __forceinline__ void load_tile_real(const PackArgs &a, int64_t r0, int64_t k0,
                                               T (*tile)[KT + 1]) {
  const int tid = threadIdx.x;
  constexpr int PER = 32 * KT / 256;
  const S *X = static_cast<const S *>(a.X) + a.Xbase;
  if (a.rfast) {
    const int rr = tid & 31, kb = tid >> 5;
    const int64_t r = pack_row(a, r0 + rr);
    const bool rok = r < a.rows;
    const int64_t ro = rok ? __ldg(a.offR + r) : 0;
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int kk = kb + 8 * i;
      const int64_t k = k0 + kk;
      const bool ok = rok && k < a.K;
      const int64_t ko = ok ? __ldg(a.offK + k) : 0;
      tile[rr][tcol<KT>(kk)] = ok ? (T)__ldg(X + ro + ko) : (T)0;
    }
  } else {
    constexpr int RSTEP = 256 / KT;
    const int kk = tid % KT, rb = tid / KT;
    const int64_t k = k0 + kk;
    const bool kok = k < a.K;
    const int64_t ko = kok ? __ldg(a.offK + k) : 0;
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int rr = rb + RSTEP * i;
      const int64_t r = pack_row(a, r0 + rr);
      const bool ok = kok && r < a.rows;
      const int64_t ro = ok ? __ldg(a.offR + r) : 0;
      tile[rr][tcol<KT>(kk)] = ok ? (T)__ldg(X + ro + ko) : (T)0;
    }
  }
}

// The same with the block's 32 row offsets and KT K offsets staged in
// shared memory first (two coalesced loads), so each element's
// load waits on a shared-memory read rather than on an offset load from
// L1/L2; every thread then issues its loads independently, coalesced along
// whichever of rows / K is X's unit-stride axis.  Every thread of the block
// calls it.  It pays in grouped launches (short blocks of many problems:
// 6 % on the 2000-block step) and loses on one large operand (the offsets
// are L1 broadcasts there and the barrier delays each block's loads: the
// pack of the permuted 4-index contraction took 0.18 ms instead of 0.12).
template <class T, class S, int KT>
__device__ __forceinline__ void load_tile_real_staged(const PackArgs &a, int64_t r0, int64_t k0,
                                                      T (*tile)[KT + 1]) {
  __shared__ int64_t s_ro[32], s_ko[KT];
  const int tid = threadIdx.x;
  constexpr int PER = 32 * KT / 256;
  for (int i = tid; i < KT; i += 256) {
    const int64_t k = k0 + i;
    s_ko[i] = k < a.K ? __ldg(a.offK + k) : INT64_MIN;
  }
  if (tid < 32) {
    const int64_t r = pack_row(a, r0 + tid);
    s_ro[tid] = r < a.rows ? a.Xbase + __ldg(a.offR + r) : INT64_MIN;
  }
  __syncthreads();
  const S *X = static_cast<const S *>(a.X);
  if (a.rfast) {
    const int rr = tid & 31, kb = tid >> 5;
    const int64_t ro = s_ro[rr];
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int kk = kb + 8 * i;
      const int64_t ko = s_ko[kk];
      const bool ok = ro != INT64_MIN && ko != INT64_MIN;
      tile[rr][tcol<KT>(kk)] = ok ? (T)__ldg(X + ro + ko) : (T)0;
    }
  } else {
    constexpr int RSTEP = 256 / KT;
    const int kk = tid % KT, rb = tid / KT;
    const int64_t ko = s_ko[kk];
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int rr = rb + RSTEP * i;
      const int64_t ro = s_ro[rr];
      const bool ok = ko != INT64_MIN && ro != INT64_MIN;
      tile[rr][tcol<KT>(kk)] = ok ? (T)__ldg(X + ro + ko) : (T)0;
    }
  }
}

template <class T, int KT>
__device__ __forceinline__ void load_tile(const PackArgs &a, int64_t r0, int64_t k0, T (*tile)[KT + 1]) {
  if (a.cmode == 0) {
    if (a.TX == QS_F64) return load_tile_real<T, double, KT>(a, r0, k0, tile);
    if (a.TX == QS_F32) return load_tile_real<T, float, KT>(a, r0, k0, tile);
  }
  const int tid = threadIdx.x;
  constexpr int PER = 32 * KT / 256;
#pragma unroll 8
  for (int i = 0; i < PER; ++i) {
    int e = tid + 256 * i, rr, kk;
    if (a.rfast) { rr = e & 31; kk = e >> 5; } else { kk = e % KT; rr = e / KT; }
    int64_t r = pack_row(a, r0 + rr), k = k0 + kk;
    T v = (T)0;
    if (r < a.rows && k < a.K) v = virtual_elem<T>(a, r, k);
    tile[rr][tcol<KT>(kk)] = v;
  }
}

// Ozaki digits of a row (the fused pack below): balanced base-256 digits.
// With E = (frexp exponent of the row's max |x|) + 1, x = v * 2^-E has
// |x| < 1/2.  The pack rounds q = x * 127/128 * 2^(8s) once to an integer,
// so |q| <= 127 * 2^(8s-8), and writes the s bytes of q + sum_i 128 * 256^i
// (each in 0..255, the sum below 2^(8s)) minus 128 as the digits d_s .. d_1:
//   v ~= 2^E * 128/127 * sum_p d_p 256^-p,
// d_1 in [-127, 127] and the others in [-128, 127], all exact int8.  The
// error is one rounding of q, at most 2^-(8s+1) * 128/127 relative to 2^E
// (base-254 digits leave (254/256)^s times that).  Rows with a NaN or Inf
// get exponent kNonFinite, zero digits, and are listed for the fixup.
constexpr double kDigitScale = 127.0 / 128.0;

// Split-BF16 planes of one 32-row x 64-element block: hi = bf16(x),
// lo = bf16(x - hi), x in FP32.
__device__ __forceinline__ void bf16_pack_block(const PackArgs &a, int64_t r0, int64_t k0) {
  __shared__ float tile[32][65];
  load_tile<float, 64>(a, r0, k0, tile);
  __syncthreads();
  const int row = threadIdx.x >> 3, c = threadIdx.x & 7;  // 8 values per chunk
  const int64_t grow = r0 + row;
  if (grow >= a.rows_pad) return;
  uint32_t hw[4], lw[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float x0 = tile[row][tcol<64>(c * 8 + 2 * q)], x1 = tile[row][tcol<64>(c * 8 + 2 * q + 1)];
    const __nv_bfloat16 h0 = __float2bfloat16_rn(x0), h1 = __float2bfloat16_rn(x1);
    const __nv_bfloat16 l0 = __float2bfloat16_rn(x0 - __bfloat162float(h0));
    const __nv_bfloat16 l1 = __float2bfloat16_rn(x1 - __bfloat162float(h1));
    hw[q] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
    lw[q] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
  }
  const int64_t off = panel_tile_base(a, grow, (k0 + c * 8) * 2);
  *reinterpret_cast<uint4 *>(a.panel + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
  *reinterpret_cast<uint4 *>(a.panel + a.plane + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
}

// Both operands of one plan in one launch (A's and B's packs are
// independent): blocks [0, nA) take A's (row block, K block) pairs, row block
// fastest, the rest B's.  Twice the blocks in flight and half the launch
// tails of one launch per operand.
__device__ __forceinline__ void split_block(int64_t b, int nrb, int64_t &r0, int64_t &kb) {
  r0 = (b % nrb) * 32;
  kb = b / nrb;
}
__global__ void __launch_bounds__(256) bf16_pack_pair_kernel(PackArgs pa, PackArgs pb, int nrbA, int nrbB,
                                                             int64_t nA) {
  int64_t r0, kb;
  const int64_t b = blockIdx.x;
  if (b < nA) {
    split_block(b, nrbA, r0, kb);
    bf16_pack_block(pa, r0, kb * 64);
  } else {
    split_block(b - nA, nrbB, r0, kb);
    bf16_pack_block(pb, r0, kb * 64);
  }
}

// Ozaki pack in two streaming passes per operand.  Pass 1 (oz_rowmax_block)
// reduces every row's max |x| bit pattern into a zeroed workspace (one
// atomicMax per row and block); pass 2 (oz_digit_block) derives the row's
// exponent from it and writes the digit planes.  Blocks are 32 rows x 128 K
// values: a thread's 16 loads are independent and in flight together, and
// six (pass 1) or four (pass 2, which holds 32 words of digit bytes per
// thread) blocks per SM keep 130-200 KB of loads outstanding.  The plan runs the
// passes operand by operand, so the second pass re-reads an operand that
// the first has just brought into L2.
constexpr int kPackRows = 32, kPackK = 128;
// Operand bytes per chunk of a grouped pack (pass 2 re-reads them from L2;
// on the 2000-block network step 48 to 160 MB measured the same, 24 MB and
// one chunk for the whole group 7 % slower).
constexpr size_t kPackChunkBytes = 96ull << 20;

// Element kinds, fixed per launch: real Float64 or real Float32 operands
// take the straight-line loads of load_tile_real; anything else (complex
// layouts, mixed types) the general loader.
enum { kPackF64 = 0, kPackF32 = 1, kPackAny = 2 };

__host__ __device__ inline int pack_kind_of(const PackArgs &a) {
  if (a.cmode == 0 && a.TX == QS_F64) return kPackF64;
  if (a.cmode == 0 && a.TX == QS_F32) return kPackF32;
  return kPackAny;
}

// STAGE: the real loaders with their offsets staged in shared memory
// (grouped launches).
template <int KIND, bool STAGE>
__device__ __forceinline__ void pack_load(const PackArgs &a, int64_t r0, int64_t k0,
                                          double (*tile)[kPackK + 1]) {
  if constexpr (KIND == kPackF64) {
    if constexpr (STAGE) load_tile_real_staged<double, double, kPackK>(a, r0, k0, tile);
    else load_tile_real<double, double, kPackK>(a, r0, k0, tile);
  } else if constexpr (KIND == kPackF32) {
    if constexpr (STAGE) load_tile_real_staged<double, float, kPackK>(a, r0, k0, tile);
    else load_tile_real<double, float, kPackK>(a, r0, k0, tile);
  } else {
    load_tile<double, kPackK>(a, r0, k0, tile);
  }
}

// Pass 1: each row's max magnitude as the bit pattern of |x| (for
// non-negative doubles the integer order is the value order, and a NaN or
// Inf sorts above every finite value).  8 threads per row.
template <int KIND, bool STAGE>
__device__ __forceinline__ void oz_rowmax_block(const PackArgs &a, int64_t r0, int64_t k0) {
  __shared__ double tile[kPackRows][kPackK + 1];
  pack_load<KIND, STAGE>(a, r0, k0, tile);
  __syncthreads();
  const int row = threadIdx.x >> 3, part = threadIdx.x & 7;
  unsigned long long m = 0;
#pragma unroll
  for (int kk = 0; kk < 16; ++kk) {
    const unsigned long long b =
        (unsigned long long)__double_as_longlong(fabs(tile[row][tcol<kPackK>(part * 16 + kk)]));
    m = b > m ? b : m;
  }
#pragma unroll
  for (int o = 1; o < 8; o <<= 1) {
    const unsigned long long x = __shfl_xor_sync(0xffffffffu, m, o);
    m = x > m ? x : m;
  }
  const int64_t r = pack_row(a, r0 + row);
  if (part == 0 && r < a.rows && m) atomicMax(a.rowmax + r, m);
}

// The row's exponent E (frexp exponent of the max + 1; kNonFinite for a row
// holding a NaN or Inf, 0 for a zero row) and digit scale
// f = 127/128 * 2^(8s - E) (wide: 127/128 * 2^(8s), after an exact scale by
// 2^-E).
struct RowScale {
  int E;
  bool bad, zero, wide;
  double f;
};
__device__ __forceinline__ RowScale row_scale(unsigned long long mb, int s) {
  RowScale r{0, mb >= 0x7FF0000000000000ull, mb == 0, false, 0.0};
  if (r.bad) {
    r.E = kNonFinite;
  } else if (!r.zero) {
    frexp(__longlong_as_double((long long)mb), &r.E);
    r.E += 1;
    const int sh = 8 * s - r.E;
    r.wide = sh < -1000 || sh > 1000;
    r.f = kDigitScale * __longlong_as_double((long long)((r.wide ? 8 * s : sh) + 1023) << 52);
  }
  return r;
}

// Pass 2: the digit planes of one 32-row x 128-K block (the balanced
// base-256 digits described above).  Thread (row, c) writes the 16 digits
// of K values c*16 .. c*16 + 15 of its row into each plane.
template <int KIND, bool STAGE>
__device__ __forceinline__ void oz_digit_block(const PackArgs &a, int64_t r0, int64_t k0) {
  __shared__ double tile[kPackRows][kPackK + 1];
  pack_load<KIND, STAGE>(a, r0, k0, tile);
  __syncthreads();
  const int row = threadIdx.x >> 3, c = threadIdx.x & 7;
  const int64_t grow = pack_row(a, r0 + row);
  if (grow >= a.rows_pad) return;
  const int s = a.nslices;
  const RowScale rs = row_scale(grow < a.rows ? __ldg(a.rowmax + grow) : 0ull, s);
  if (k0 == 0 && c == 0) {
    a.exp_out[grow] = rs.E;
    if (rs.bad) a.flag_list[atomicAdd(a.flag_count, 1)] = (int32_t)grow;
  }
  // q = the value times f rounded once to an integer, |q| <= 127 * 2^(8s-8);
  // the bytes of q + 0x80..80 (s bytes) are the digits + 128, low digit
  // first.  For s <= 6, |q| < 2^47: one FMA with 1.5 * 2^52 rounds the exact
  // v * f to q (ties to even) and leaves 2^51 + q in the low 52 bits of its
  // bit pattern, so the low 8s bits of those bits + (bias - 2^51) are
  // q + bias.  s = 7 needs 56 bits and converts.
  const unsigned long long bias = 0x8080808080808080ull >> (64 - 8 * s);
  constexpr double kMagic = 6755399441055744.0;  // 1.5 * 2^52
  const unsigned long long mbias = bias - (1ull << 51);
  const bool live = !rs.bad && !rs.zero;
  uint32_t lo[16], hi[16];
#pragma unroll
  for (int kk = 0; kk < 16; ++kk) {
    unsigned long long u = bias;  // the digits of 0
    if (live) {
      const double v = tile[row][tcol<kPackK>(c * 16 + kk)];
      if (s <= 6) {
        const double t = rs.wide ? __dadd_rn(__dmul_rn(scale2(v, -rs.E), rs.f), kMagic) : __fma_rn(v, rs.f, kMagic);
        u = (unsigned long long)__double_as_longlong(t) + mbias;
      } else {
        const double y = rs.wide ? scale2(v, -rs.E) * rs.f : v * rs.f;
        u = (unsigned long long)__double2ll_rn(y) + bias;
      }
    }
    lo[kk] = (uint32_t)u;
    hi[kk] = (uint32_t)(u >> 32);
  }
  uint8_t *dst = a.panel + panel_tile_base(a, grow, k0 + c * 16);
  const int64_t plane = a.plane;
  for (int p = 0; p < s; ++p) {
    // plane p holds digit p + 1 (weight 256^-(p+1)): byte s - 1 - p of q + bias
    const int bi = s - 1 - p;
    const uint32_t sel = 0x11u * (uint32_t)(bi & 3) + 0x40u;  // byte bi of x, byte bi of y
    uint32_t wd[4];
    if (bi >= 4) {
#pragma unroll
      for (int j = 0; j < 4; ++j)
        wd[j] = __byte_perm(__byte_perm(hi[4 * j], hi[4 * j + 1], sel), __byte_perm(hi[4 * j + 2], hi[4 * j + 3], sel),
                            0x5410) ^ 0x80808080u;
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j)
        wd[j] = __byte_perm(__byte_perm(lo[4 * j], lo[4 * j + 1], sel), __byte_perm(lo[4 * j + 2], lo[4 * j + 3], sel),
                            0x5410) ^ 0x80808080u;
    }
    *reinterpret_cast<uint4 *>(dst + p * plane) = make_uint4(wd[0], wd[1], wd[2], wd[3]);
  }
}

// One operand of one plan: blocks (row block fastest, then K block).
__device__ __forceinline__ void pack_block_coords(int64_t b, int nrb, int64_t &r0, int64_t &k0) {
  r0 = (b % nrb) * kPackRows;
  k0 = (b / nrb) * kPackK;
}

template <int KIND>
__global__ void __launch_bounds__(256, 6) oz_rowmax_kernel(const __grid_constant__ PackArgs a, int nrb) {
  int64_t r0, k0;
  pack_block_coords(blockIdx.x, nrb, r0, k0);
  oz_rowmax_block<KIND, false>(a, r0, k0);
}

template <int KIND>
__global__ void __launch_bounds__(256, 4) oz_digit_kernel(const __grid_constant__ PackArgs a, int nrb) {
  int64_t r0, k0;
  pack_block_coords(blockIdx.x, nrb, r0, k0);
  oz_digit_block<KIND, false>(a, r0, k0);
}

// Pass 1 and pass 2 of one operand: blocks cover rows_pad x kblocks * 128
// (pass 1 only needs K, pass 2 writes the zero padding of K too).
static cudaError_t launch_pack_operand(const PackArgs &a, cudaStream_t st) {
  const int nrb = (int)((a.rows_pad + kPackRows - 1) / kPackRows);
  const unsigned n1 = (unsigned)((int64_t)nrb * ((a.K + kPackK - 1) / kPackK));
  const unsigned n2 = (unsigned)((int64_t)nrb * a.kblocks);
  switch (pack_kind_of(a)) {
    case kPackF64:
      oz_rowmax_kernel<kPackF64><<<n1, 256, 0, st>>>(a, nrb);
      oz_digit_kernel<kPackF64><<<n2, 256, 0, st>>>(a, nrb);
      break;
    case kPackF32:
      oz_rowmax_kernel<kPackF32><<<n1, 256, 0, st>>>(a, nrb);
      oz_digit_kernel<kPackF32><<<n2, 256, 0, st>>>(a, nrb);
      break;
    default:
      oz_rowmax_kernel<kPackAny><<<n1, 256, 0, st>>>(a, nrb);
      oz_digit_kernel<kPackAny><<<n2, 256, 0, st>>>(a, nrb);
      break;
  }
  return cudaGetLastError();
}

// ---------------------------------------------------------------- GEMM ---

enum { KIND_I8 = 0, KIND_BF16 = 1 };
// K values per FP32-accumulated segment of a BF16x3 tile (4 K blocks).
constexpr int kBf16SegK = 256;

struct GemmArgs {
  const uint8_t *panelA, *panelB;
  int64_t planeA, planeB;
  int mtiles, ntiles, kblocks;
  int nslices;       // Ozaki slices (I8)
  int kseg_blocks;   // K blocks per INT32-exact segment (I8)
  int nkseg;         // K segments per diagonal (I8)
  const int32_t *expA, *expB;
  void *C;
  int64_t Cbase;
  int TC;
  const int64_t *offMC, *offNC;
  int64_t M, N;
  double alpha, beta;
  double alpha_im, beta_im;
  int beta_case;
  int cplx;  // 0 real; 1 = 1m: real rows 2i / 2i+1 are Re / Im of complex
             // row i; 2 = planar: real columns 2n / 2n+1 are Re / Im of n
  int *status;
  double wdiag[16];  // weight of diagonal t (Ozaki): (128/127)^2 256^-(t+2)
  uint64_t wait_ns;  // bound of every barrier wait (qs_plan_set_wait_limit)
  int hold_loads;    // failure-detection test: the producers issue no copies
  int band_m;        // tile raster: m-tiles per band (Ozaki kernels)
};

// The alpha/beta store of one 16-column chunk of a row of the tile, values
// in the compute precision R.  Ozaki values are rescaled by 2^(eA + eB) first.
// Complex (1m): lanes 2l and 2l+1 hold Re and Im of one complex element; the
// pair is joined with a shuffle and the even lane stores it.
// Any C eltype, real or complex (1m lane pairs).
template <class R>
__device__ __forceinline__ void store_chunk_any(const GemmArgs &a, const R (&v)[16], int c, int64_t n0,
                                                bool row_store, int64_t crow, int lane,
                                                const int64_t *s_offN, const int32_t *s_expN, int eA) {
  constexpr int kNF = INT_MIN;
  constexpr int G = 2;  // old C values in flight per thread (register budget)
  auto prep = [&](int e, R &x, int64_t &idx) -> bool {
    const int jj = 16 * c + e;
    const int eB = s_expN[jj];
    const bool finite = eA != kNF && eB != kNF;
    x = v[e];
    if (sizeof(R) == 8 && finite) x = (R)scale2((double)x, eA + eB);
    idx = crow + s_offN[jj];
    return row_store && n0 + jj < a.N && finite;
  };
  if (a.cplx == 2) {
    // planar: columns 16c + 2u and 16c + 2u + 1 are Re and Im of one element
    Scalars<cplx<R>> s;
    s.alpha.re = (R)a.alpha; s.alpha.im = (R)a.alpha_im;
    s.beta.re = (R)a.beta; s.beta.im = (R)a.beta_im;
    s.beta_case = a.beta_case;
#pragma unroll
    for (int e0 = 0; e0 < 16; e0 += 2 * G) {
      cplx<R> old[G];
#pragma unroll
      for (int u = 0; u < G; ++u) {
        R x;
        int64_t idx;
        const bool ok = prep(e0 + 2 * u, x, idx);
        old[u] = (ok && a.beta_case != 0) ? load_c<cplx<R>>(a.C, idx, a.TC) : tzero<cplx<R>>();
      }
#pragma unroll
      for (int u = 0; u < G; ++u) {
        R xr, xi;
        int64_t idx, idx2;
        const bool ok = prep(e0 + 2 * u, xr, idx);
        prep(e0 + 2 * u + 1, xi, idx2);
        if (ok) {
          cplx<R> r;
          r.re = xr;
          r.im = xi;
          store_c<cplx<R>>(a.C, idx, a.TC, axpby(s, r, old[u]));
        }
      }
    }
  } else if (a.cplx) {
    Scalars<cplx<R>> s;
    s.alpha.re = (R)a.alpha; s.alpha.im = (R)a.alpha_im;
    s.beta.re = (R)a.beta; s.beta.im = (R)a.beta_im;
    s.beta_case = a.beta_case;
#pragma unroll
    for (int e0 = 0; e0 < 16; e0 += G) {
      cplx<R> old[G];
#pragma unroll
      for (int e = 0; e < G; ++e) {
        R x;
        int64_t idx;
        const bool ok = prep(e0 + e, x, idx) && (lane & 1) == 0;
        old[e] = (ok && a.beta_case != 0) ? load_c<cplx<R>>(a.C, idx, a.TC) : tzero<cplx<R>>();
      }
#pragma unroll
      for (int e = 0; e < G; ++e) {
        R x;
        int64_t idx;
        const bool ok = prep(e0 + e, x, idx);
        const R other = __shfl_xor_sync(0xffffffffu, x, 1);
        if (ok && (lane & 1) == 0) {
          cplx<R> r;
          r.re = x;
          r.im = other;
          store_c<cplx<R>>(a.C, idx, a.TC, axpby(s, r, old[e]));
        }
      }
    }
  } else {
    Scalars<R> s;
    s.alpha = (R)a.alpha;
    s.beta = (R)a.beta;
    s.beta_case = a.beta_case;
#pragma unroll
    for (int e0 = 0; e0 < 16; e0 += G) {
      R old[G];
#pragma unroll
      for (int e = 0; e < G; ++e) {
        R x;
        int64_t idx;
        const bool ok = prep(e0 + e, x, idx);
        old[e] = (ok && a.beta_case != 0) ? load_c<R>(a.C, idx, a.TC) : (R)0;
      }
#pragma unroll
      for (int e = 0; e < G; ++e) {
        R x;
        int64_t idx;
        if (prep(e0 + e, x, idx)) store_c<R>(a.C, idx, a.TC, axpby(s, x, old[e]));
      }
    }
  }
}

// Real FP64 C: the compact path.  Old C values are loaded G at a time
// before their stores, so the loads overlap.
__device__ __forceinline__ void store_chunk_f64(const GemmArgs &a, const double (&v)[16], int c,
                                                int64_t n0, bool row_store, int64_t crow,
                                                const int64_t *s_offN, const int32_t *s_expN,
                                                int eA) {
  constexpr int kNF = INT_MIN;
  constexpr int G = 4;
  double *C = static_cast<double *>(a.C);
  const double al = a.alpha, be = a.beta;
  const int bc = a.beta_case;
#pragma unroll
  for (int e0 = 0; e0 < 16; e0 += G) {
    double old[G];
#pragma unroll
    for (int e = 0; e < G; ++e) {
      const int jj = 16 * c + e0 + e;
      const bool ok = row_store && n0 + jj < a.N && s_expN[jj] != kNF;
      old[e] = (ok && bc != 0) ? C[crow + s_offN[jj]] : 0.0;
    }
#pragma unroll
    for (int e = 0; e < G; ++e) {
      const int jj = 16 * c + e0 + e;
      const int eB = s_expN[jj];
      if (!row_store || n0 + jj >= a.N || eB == kNF) continue;
      const double x = scale2(v[e0 + e], eA + eB);
      double r;
      if (bc == 0) r = al * x;
      else if (bc == 1) r = fma(al, x, old[e]);
      else r = fma(al, x, be * old[e]);
      C[crow + s_offN[jj]] = r;
    }
  }
}

// Real FP64 C takes the compact path.
__device__ __forceinline__ bool store_is_f64(const GemmArgs &a) { return !a.cplx && a.TC == QS_F64; }

template <class R>
__device__ __forceinline__ void store_chunk(const GemmArgs &a, const R (&v)[16], int c, int64_t n0,
                                            bool row_store, int64_t crow, int lane,
                                            const int64_t *s_offN, const int32_t *s_expN, int eA) {
  if constexpr (sizeof(R) == 8) {
    if (store_is_f64(a)) {
      store_chunk_f64(a, v, c, n0, row_store, crow, s_offN, s_expN, eA);
      return;
    }
  }
  store_chunk_any<R>(a, v, c, n0, row_store, crow, lane, s_offN, s_expN, eA);
}

// L2 prefetch of the C elements this thread will read back in its final
// store (beta != 0): issued when the tile starts, long before the store.
__device__ __forceinline__ void prefetch_c_row(const GemmArgs &a, int64_t crow, const int64_t *s_offN,
                                               int j0, int nj, int64_t n0) {
  if (a.beta_case == 0) return;
  const int es = (a.TC == QS_F32) ? 4 : (a.TC == QS_C64 ? 16 : 8);
  const char *base = static_cast<const char *>(a.C);
  for (int j = j0; j < j0 + nj; ++j) {
    if (n0 + j >= a.N) break;
    const char *p = base + (crow + s_offN[j]) * es;
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
  }
}

template <int KIND>
struct GemmCfg;
template <>
struct GemmCfg<KIND_I8> {
  static constexpr int BN = 128, STAGES = 6, KSTEP_BYTES = 32;
  static constexpr uint32_t IDESC = idesc_i8(128, 128);
};
template <>
struct GemmCfg<KIND_BF16> {
  static constexpr int BN = 128, STAGES = 6, KSTEP_BYTES = 32;
  static constexpr uint32_t IDESC = idesc_bf16(128, 128);
};

template <int KIND>
constexpr size_t gemm_smem_bytes() {
  using Cfg = GemmCfg<KIND>;
  return 1024 + (size_t)Cfg::STAGES * (kTileM * kKBytes + Cfg::BN * kKBytes) + 1024 +
         Cfg::BN * (sizeof(int64_t) + sizeof(int32_t));
}

// C offsets of real (virtual) row i and real column n of the GEMM.
__device__ __forceinline__ int64_t c_row(const GemmArgs &a, int64_t i) {
  return a.offMC[a.cplx == 1 ? (i >> 1) : i];
}
__device__ __forceinline__ int64_t c_col(const GemmArgs &a, int64_t n) {
  return a.offNC[a.cplx == 2 ? (n >> 1) : n];
}

// The problem table of a grouped launch: tile t of the launch belongs to
// problem p when tile_start[p] <= t < tile_start[p + 1].  nprob == 0 means a
// single problem, the kernel's own GemmArgs.
struct GemmTable {
  const GemmArgs *tab;
  const int *tile_start;
  const int *tile_prob;  // problem of each tile of the launch
  int nprob;
};

template <bool GROUPED>
__device__ __forceinline__ const GemmArgs &tile_problem(const GemmArgs &a, const GemmTable &g, int t,
                                                        int &local) {
  if (!GROUPED) {
    local = t;
    return a;
  }
  const int p = __ldg(g.tile_prob + t);
  local = t - __ldg(g.tile_start + p);
  return g.tab[p];
}

// Segments of a tile: Ozaki, one per (diagonal, K segment); BF16x3, one per
// K segment (FP32 accumulation over at most kBf16SegK K values, the
// segments summed in FP64).
__device__ __forceinline__ int seg_count(const GemmArgs &a, int kind) {
  return kind == KIND_I8 ? a.nslices * a.nkseg : a.nkseg;
}
// Terms of segment g: (plane of A, plane of B) for term index j, and the K
// block range.
__device__ __forceinline__ int seg_terms(const GemmArgs &a, int kind, int g) {
  return kind == KIND_I8 ? (g / a.nkseg) + 1 : 3;
}
__device__ __forceinline__ void seg_term(const GemmArgs &a, int kind, int g, int j, int &pa, int &pb) {
  if (kind == KIND_I8) {
    int t = g / a.nkseg;
    pa = j;
    pb = t - j;
  } else {
    pa = (j == 2) ? 1 : 0;  // (hi,hi), (hi,lo), (lo,hi)
    pb = (j == 1) ? 1 : 0;
  }
}
__device__ __forceinline__ void seg_krange(const GemmArgs &a, int kind, int g, int &kb0, int &kb1) {
  const int ks = g % a.nkseg;
  kb0 = ks * a.kseg_blocks;
  kb1 = min(kb0 + a.kseg_blocks, a.kblocks);
}

template <int KIND>
__global__ void __launch_bounds__(192, 1) tc_gemm_kernel(const __grid_constant__ GemmArgs a, const GemmTable gt) {
  using Cfg = GemmCfg<KIND>;
  constexpr int BN = Cfg::BN, STAGES = Cfg::STAGES;
  constexpr uint32_t A_BYTES = kTileM * kKBytes, B_BYTES = BN * kKBytes;
  constexpr int KSTEPS = kKBytes / Cfg::KSTEP_BYTES;
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t *sA = smem;
  uint8_t *sB = smem + STAGES * A_BYTES;
  uint64_t *bars = (uint64_t *)(sB + STAGES * B_BYTES);
  uint64_t *full = bars, *empty = bars + STAGES, *accf = bars + 2 * STAGES, *acce = accf + 2;
  uint64_t *drainb = acce + 2;  // the MMA thread's exit drain
  uint32_t *tmem_slot = (uint32_t *)(drainb + 1);
  volatile int *abort = (volatile int *)(tmem_slot + 1);
  int64_t *s_offN = (int64_t *)(smem + STAGES * (A_BYTES + B_BYTES) + 1024);
  int32_t *s_expN = (int32_t *)(s_offN + BN);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], 4);
    }
    mbar_init(drainb, 1);
    *abort = 0;
    fence_mbar_init();
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int ntile_total = gt.nprob ? gt.tile_start[gt.nprob] : a.mtiles * a.ntiles;
  uint32_t issued = 0;  // the producer's fills, in ring order (the exit drain's count)

  if (warp == 0) {
    // ---------------------------------------------------- producer ----
    if (lane == 0) {
      uint32_t stage = 0, phase = 0;
      for (int tile = blockIdx.x; tile < ntile_total && !a.hold_loads; tile += gridDim.x) {
        int lt;
        const GemmArgs &P = gt.nprob ? tile_problem<true>(a, gt, tile, lt) : tile_problem<false>(a, gt, tile, lt);
        const int mt = lt / P.ntiles, nt = lt % P.ntiles;
        const int nseg = seg_count(P, KIND);
        for (int g = 0; g < nseg; ++g) {
          int kb0, kb1;
          seg_krange(P, KIND, g, kb0, kb1);
          const int nt_terms = seg_terms(P, KIND, g);
          for (int j = 0; j < nt_terms; ++j) {
            int pa, pb;
            seg_term(P, KIND, g, j, pa, pb);
            const uint8_t *srcA = P.panelA + pa * P.planeA + ((int64_t)mt * P.kblocks) * A_BYTES;
            const uint8_t *srcB = P.panelB + pb * P.planeB + ((int64_t)nt * P.kblocks) * B_BYTES;
            for (int kb = kb0; kb < kb1; ++kb) {
              if (!mbar_wait(&empty[stage], phase ^ 1, abort, a.status, QS_ETIMEOUT, a.wait_ns)) goto done;
              mbar_arrive_expect_tx(&full[stage], A_BYTES + B_BYTES);
              bulk_g2s(sA + stage * A_BYTES, srcA + (int64_t)kb * A_BYTES, A_BYTES, &full[stage]);
              bulk_g2s(sB + stage * B_BYTES, srcB + (int64_t)kb * B_BYTES, B_BYTES, &full[stage]);
              ++issued;
              if (++stage == STAGES) {
                stage = 0;
                phase ^= 1;
              }
            }
          }
        }
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------------- MMA ------
    if (lane == 0) {
      uint32_t stage = 0, phase = 0, sc = 0;
      for (int tile = blockIdx.x; tile < ntile_total; tile += gridDim.x) {
        int lt;
        const GemmArgs &P = gt.nprob ? tile_problem<true>(a, gt, tile, lt) : tile_problem<false>(a, gt, tile, lt);
        const int nseg = seg_count(P, KIND);
        for (int g = 0; g < nseg; ++g, ++sc) {
          const uint32_t buf = sc & 1, ap = (sc >> 1) & 1;
          if (!mbar_wait(&acce[buf], ap ^ 1, abort, a.status, QS_ETIMEOUT, a.wait_ns)) goto done;
          tc_fence_after();
          const uint32_t d = tmem + buf * BN;
          int kb0, kb1;
          seg_krange(P, KIND, g, kb0, kb1);
          const int nt_terms = seg_terms(P, KIND, g);
          uint32_t acc = 0;
          for (int j = 0; j < nt_terms; ++j) {
            for (int kb = kb0; kb < kb1; ++kb) {
              if (!mbar_wait(&full[stage], phase, abort, a.status, QS_ETIMEOUT, a.wait_ns)) goto done;
              tc_fence_after();
              const uint32_t a0 = smem_u32(sA + stage * A_BYTES), b0 = smem_u32(sB + stage * B_BYTES);
#pragma unroll
              for (int ks = 0; ks < KSTEPS; ++ks) {
                const uint64_t ad = sw128_kmajor_desc(a0 + ks * Cfg::KSTEP_BYTES);
                const uint64_t bd = sw128_kmajor_desc(b0 + ks * Cfg::KSTEP_BYTES);
                if (KIND == KIND_I8) mma_i8(d, ad, bd, Cfg::IDESC, acc);
                else mma_f16(d, ad, bd, Cfg::IDESC, acc);
                acc = 1;
              }
              tc_commit(&empty[stage]);
              if (++stage == STAGES) {
                stage = 0;
                phase ^= 1;
              }
            }
          }
          tc_commit(&accf[buf]);
        }
      }
    }
  } else {
    // --------------------------------------------------- epilogue -----
    const int q = warp & 3;           // TMEM lane quarter of this warp
    const int et = threadIdx.x - 64;  // 0..127
    const uint32_t lane_base = (uint32_t)(32 * q) << 16;
    uint32_t sc = 0;
    for (int tile = blockIdx.x; tile < ntile_total; tile += gridDim.x) {
      int lt;
      const GemmArgs &P = gt.nprob ? tile_problem<true>(a, gt, tile, lt) : tile_problem<false>(a, gt, tile, lt);
      const int mt = lt / P.ntiles, nt = lt % P.ntiles;
      const int nseg = seg_count(P, KIND);
      const int64_t m0 = (int64_t)mt * kTileM, n0 = (int64_t)nt * BN;
      named_bar_sync(1, 128);
      for (int j = et; j < BN; j += 128) {
        int64_t n = n0 + j;
        s_offN[j] = n < P.N ? c_col(P, n) : 0;
        s_expN[j] = (KIND == KIND_I8 && n < P.N) ? P.expB[n] : 0;
      }
      named_bar_sync(1, 128);
      const int64_t i = m0 + 32 * q + lane;  // real (virtual) row
      const bool row_ok = i < P.M;
      const int eA = (KIND == KIND_I8 && row_ok) ? P.expA[i] : 0;
      const int64_t crow = row_ok ? P.Cbase + c_row(P, i) : 0;
      const bool row_store = row_ok && eA != kNonFinite;
      for (int g = 0; g < nseg; ++g, ++sc) {
        const uint32_t buf = sc & 1, ap = (sc >> 1) & 1;
        if (!mbar_wait(&accf[buf], ap, abort, P.status, QS_ETIMEOUT, a.wait_ns)) goto done;
        tc_fence_after();
        const bool first = (g == 0), last = (g == nseg - 1);
        const uint32_t tacc = tmem + lane_base + buf * BN;
        const uint32_t tsum = tmem + lane_base + 256;
        const double w = KIND == KIND_I8 ? P.wdiag[g / P.nkseg] : 1.0;
#pragma unroll 1
        for (int c = 0; c < BN / 16; ++c) {
          uint32_t dr[16], sr[32];
          tmem_ld16(tacc + 16 * c, dr);
          if (!first) {
            tmem_ld16(tsum + 32 * c, sr);
            tmem_ld16(tsum + 32 * c + 16, sr + 16);
          }
          tmem_ld_wait();
          double v[16];
#pragma unroll
          for (int e = 0; e < 16; ++e) {
            const double s0 = first ? 0.0 : __hiloint2double((int)sr[2 * e + 1], (int)sr[2 * e]);
            const double x = KIND == KIND_I8 ? (double)(int32_t)dr[e] : (double)__uint_as_float(dr[e]);
            v[e] = fma(x, w, s0);
          }
          if (!last) {
#pragma unroll
            for (int e = 0; e < 16; ++e) {
              sr[2 * e] = (uint32_t)__double2loint(v[e]);
              sr[2 * e + 1] = (uint32_t)__double2hiint(v[e]);
            }
            tmem_st16(tsum + 32 * c, sr);
            tmem_st16(tsum + 32 * c + 16, sr + 16);
          } else {
            store_chunk<double>(P, v, c, n0, row_store, crow, lane, s_offN, s_expN, eA);
          }
        }
        if (!last) tmem_st_wait();
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&acce[buf]);
      }
    }
  }
done:
  // Before TMEM is released and the CTA exits: every copy the producer issued
  // has landed and every MMA is complete (instant after a normal run).
  if (warp == 0 && lane == 0) drain_ring(full, STAGES, issued, a.status, a.wait_ns);
  if (warp == 1 && lane == 0) {
    tc_commit(drainb);
    mbar_wait_drain(drainb, 0, a.status, a.wait_ns);
  }
  __syncwarp();
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// ------------------------------------------------------ Ozaki GEMM (v2) ---
// Slice products grouped so each slice tile is fetched once per K block and
// group instead of once per product.  Diagonals t = p+q are taken in groups
// of up to four ({0..3}, {4..7}); every diagonal of a group has its own INT32
// accumulator (4 x 128 TMEM columns), and the FP64 running sum lives in the
// registers of eight epilogue warps (64 doubles per thread: one row, one
// half of the 128 columns).  Per K block a group loads its B slices as a
// sliding window and streams A_p once; 16 KB tiles move through a ring of
// kOzSlots shared-memory slots, each freed by the commit after its last MMA.

constexpr int kOzSlots = 13;
constexpr int kOzMaxLoads = 16, kOzMaxSteps = 40;

struct OzGroup {
  int t0, t1;  // diagonal range of the group
  int nloads, nsteps;
  int8_t load_side[kOzMaxLoads], load_slice[kOzMaxLoads];  // side 0 = A, 1 = B
  int8_t step_a[kOzMaxSteps], step_b[kOzMaxSteps], step_acc[kOzMaxSteps];
  uint16_t step_free[kOzMaxSteps];  // loads whose last use is this step
};
struct OzSched {
  int ngroups;
  OzGroup g[2];
};

struct GMeta {
  int nloads, nsteps, t0, t1;
};

constexpr size_t oz_smem_bytes() {
  return 1024 + (size_t)kOzSlots * 16384 + 1024 + 128 * (sizeof(int64_t) + sizeof(int32_t)) +
         1024;  // the schedule, staged from the parameters
}

// 10 warps: two of the four SM sub-partitions hold three warps, which caps a
// thread at 168 registers (the launch bound below).
__global__ void __launch_bounds__(320, 1)
    oz_gemm_kernel(const __grid_constant__ GemmArgs a, const __grid_constant__ OzSched sch) {
  constexpr uint32_t TILE = 128 * 128;
  constexpr uint32_t IDESC = idesc_i8(128, 128);
  extern __shared__ uint8_t smem_raw[];
  uint8_t *smem = (uint8_t *)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t *slots = smem;
  uint64_t *bars = (uint64_t *)(slots + kOzSlots * TILE);
  uint64_t *full = bars, *empty = bars + kOzSlots, *accf = bars + 2 * kOzSlots, *acce = accf + 4;
  uint64_t *drainb = acce + 4;  // the MMA thread's exit drain
  uint32_t *tmem_slot = (uint32_t *)(drainb + 1);
  volatile int *abort = (volatile int *)(tmem_slot + 1);
  int64_t *s_offN = (int64_t *)(smem + kOzSlots * TILE + 1024);
  int32_t *s_expN = (int32_t *)(s_offN + 128);
  // The schedule in shared memory: one word per product step (load of A in
  // bits 0-3, load of B in 4-7, accumulator in 8-9, loads freed after the
  // step in 16-31) and one byte per load (side << 4 | slice).  Read with
  // dynamic indices in the issue loops, parameters would go through the
  // slow load path on every step.
  uint32_t *s_step = (uint32_t *)(s_expN + 128);        // [2][kOzMaxSteps]
  uint8_t *s_load = (uint8_t *)(s_step + 2 * kOzMaxSteps);  // [2][kOzMaxLoads]
  GMeta *s_meta = (GMeta *)(s_load + 2 * kOzMaxLoads);      // [2]

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < kOzSlots; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 4; ++b) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], 8);
    }
    mbar_init(drainb, 1);
    *abort = 0;
    fence_mbar_init();
    for (int gi = 0; gi < sch.ngroups; ++gi) {
      const OzGroup &Gp = sch.g[gi];
      s_meta[gi] = GMeta{Gp.nloads, Gp.nsteps, Gp.t0, Gp.t1};
      const OzGroup &G = Gp;
      for (int st = 0; st < G.nsteps; ++st)
        s_step[gi * kOzMaxSteps + st] = (uint32_t)(G.step_a[st] & 15) | ((uint32_t)(G.step_b[st] & 15) << 4) |
                                        ((uint32_t)(G.step_acc[st] & 3) << 8) |
                                        ((uint32_t)G.step_free[st] << 16);
      for (int l = 0; l < G.nloads; ++l)
        s_load[gi * kOzMaxLoads + l] = (uint8_t)((G.load_side[l] << 4) | (G.load_slice[l] & 15));
    }
  }
  if (warp == 1) {
    tmem_alloc(tmem_slot, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int ntile_total = a.mtiles * a.ntiles;
  uint32_t issued = 0;  // the producer's fills, in ring order (the exit drain's count)

  if (warp == 0) {
    // ---------------------------------------------------- producer ----
    if (lane == 0) {
      uint32_t L = 0;
      for (int tile = blockIdx.x; tile < ntile_total && !a.hold_loads; tile += gridDim.x) {
        const int mt = tile / a.ntiles, nt = tile % a.ntiles;
        for (int gi = 0; gi < sch.ngroups; ++gi) {
          const GMeta G = s_meta[gi];
          for (int ks = 0; ks < a.nkseg; ++ks) {
            const int kb0 = ks * a.kseg_blocks, kb1 = min(kb0 + a.kseg_blocks, a.kblocks);
            for (int kb = kb0; kb < kb1; ++kb) {
              for (int l = 0; l < G.nloads; ++l, ++L) {
                const uint32_t slot = L % kOzSlots, round = L / kOzSlots;
                if (!mbar_wait(&empty[slot], (round & 1) ^ 1, abort, a.status, QS_ETIMEOUT, a.wait_ns)) goto done;
                mbar_arrive_expect_tx(&full[slot], TILE);
                const int code = s_load[gi * kOzMaxLoads + l];
                const uint8_t *src =
                    (code >> 4) == 0
                        ? a.panelA + (code & 15) * a.planeA + ((int64_t)mt * a.kblocks + kb) * TILE
                        : a.panelB + (code & 15) * a.planeB + ((int64_t)nt * a.kblocks + kb) * TILE;
                bulk_g2s(slots + slot * TILE, src, TILE, &full[slot]);
                ++issued;
              }
            }
          }
        }
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------------- MMA ------
    if (lane == 0) {
      uint32_t L = 0;
      uint32_t accpar = 0;  // bit q: parity of accumulator q's use count
      for (int tile = blockIdx.x; tile < ntile_total; tile += gridDim.x) {
        for (int gi = 0; gi < sch.ngroups; ++gi) {
          const GMeta G = s_meta[gi];
          const int nacc = G.t1 - G.t0 + 1;
          for (int ks = 0; ks < a.nkseg; ++ks) {
            for (int q = 0; q < nacc; ++q)
              if (!mbar_wait(&acce[q], ((accpar >> q) & 1u) ^ 1u, abort, a.status, QS_ETIMEOUT, a.wait_ns)) goto done;
            tc_fence_after();
            uint32_t started = 0;
            const int kb0 = ks * a.kseg_blocks, kb1 = min(kb0 + a.kseg_blocks, a.kblocks);
            for (int kb = kb0; kb < kb1; ++kb) {
              const uint32_t base = L;
              uint32_t waited = 0;
              for (int st = 0; st < G.nsteps; ++st) {
                const uint32_t word = s_step[gi * kOzMaxSteps + st];
                const int la = word & 15, lb = (word >> 4) & 15;
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                  const int l = u ? lb : la;
                  if (!((waited >> l) & 1u)) {
                    const uint32_t gl = base + l;
                    if (!mbar_wait(&full[gl % kOzSlots], (gl / kOzSlots) & 1, abort, a.status, QS_ETIMEOUT,
                                   a.wait_ns))
                      goto done;
                    waited |= 1u << l;
                  }
                }
                tc_fence_after();
                const int acc = (word >> 8) & 3;
                const uint32_t d = tmem + acc * 128;
                const uint32_t a0 = smem_u32(slots + ((base + la) % kOzSlots) * TILE);
                const uint32_t b0 = smem_u32(slots + ((base + lb) % kOzSlots) * TILE);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                  const uint32_t accum = (((started >> acc) & 1u) || j > 0) ? 1u : 0u;
                  mma_i8(d, sw128_kmajor_desc(a0 + 32 * j), sw128_kmajor_desc(b0 + 32 * j), IDESC, accum);
                }
                started |= 1u << acc;
                uint32_t fr = word >> 16;
                while (fr) {
                  const int l = __ffs(fr) - 1;
                  fr &= fr - 1;
                  tc_commit(&empty[(base + l) % kOzSlots]);
                }
              }
              L += G.nloads;
            }
            for (int q = 0; q < nacc; ++q) {
              tc_commit(&accf[q]);
              accpar ^= 1u << q;
            }
          }
        }
      }
    }
  } else {
    // --------------------------------------------------- epilogue -----
    const int q = warp & 3;               // TMEM lane quarter
    const int h = (warp - 2) >> 2;        // column half: 0 or 1
    const int et = threadIdx.x - 64;      // 0..255
    const uint32_t lane_base = (uint32_t)(32 * q) << 16;
    uint32_t accpar = 0;  // bit q: parity of accumulator q's use count
    double sum[64];
    for (int tile = blockIdx.x; tile < ntile_total; tile += gridDim.x) {
      const int mt = tile / a.ntiles, nt = tile % a.ntiles;
      const int64_t m0 = (int64_t)mt * 128, n0 = (int64_t)nt * 128;
      named_bar_sync(1, 256);
      if (et < 128) {
        const int64_t n = n0 + et;
        s_offN[et] = n < a.N ? c_col(a, n) : 0;
        s_expN[et] = n < a.N ? a.expB[n] : 0;
      }
      named_bar_sync(1, 256);
      const int64_t i = m0 + 32 * q + lane;
      const bool row_ok = i < a.M;
      const int eA = row_ok ? a.expA[i] : 0;
      const int64_t crow = row_ok ? a.Cbase + c_row(a, i) : 0;
      const bool row_store = row_ok && eA != kNonFinite;
      bool first = true;
      for (int gi = 0; gi < sch.ngroups; ++gi) {
        const GMeta G = s_meta[gi];
        const int nacc = G.t1 - G.t0 + 1;
        for (int ks = 0; ks < a.nkseg; ++ks) {
          for (int qa = 0; qa < nacc; ++qa) {
            if (!mbar_wait(&accf[qa], (accpar >> qa) & 1u, abort, a.status, QS_ETIMEOUT, a.wait_ns)) goto done;
            tc_fence_after();
            const double w = a.wdiag[G.t0 + qa];
            const uint32_t taddr = tmem + lane_base + qa * 128 + 64 * h;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
              uint32_t dr[16];
              tmem_ld16(taddr + 16 * c, dr);
              tmem_ld_wait();
#pragma unroll
              for (int e = 0; e < 16; ++e)
                sum[16 * c + e] = fma((double)(int32_t)dr[e], w, first ? 0.0 : sum[16 * c + e]);
            }
            first = false;
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acce[qa]);
            accpar ^= 1u << qa;
          }
        }
      }
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        double v[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) v[e] = sum[16 * c + e];
        store_chunk<double>(a, v, 4 * h + c, n0, row_store, crow, lane, s_offN, s_expN, eA);
      }
    }
  }
done:
  // Before TMEM is released and the CTA exits: every copy the producer issued
  // has landed and every MMA is complete (instant after a normal run).
  if (warp == 0 && lane == 0) drain_ring(full, kOzSlots, issued, a.status, a.wait_ns);
  if (warp == 1 && lane == 0) {
    tc_commit(drainb);
    mbar_wait_drain(drainb, 0, a.status, a.wait_ns);
  }
  __syncwarp();
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    tmem_dealloc(tmem, 512);
  }
}

// ------------------------------------------- Ozaki GEMM, fixed schedule ---
// The v2 kernel with the schedule a compile-time constant (one instance per
// slice count): the issue loops unroll into straight-line code, so a product
// step is its barrier waits (only where a tile is first used), four MMAs and
// the commits of the tiles it frees.  One thread issues every MMA, so its
// per-step instruction count bounds the tensor pipe.

template <int S>
struct OzFixedSched {
  struct Grp {
    int t0, t1, nloads, nsteps;
    int side[kOzMaxLoads], slice[kOzMaxLoads], first_use[kOzMaxLoads];
    int sa[kOzMaxSteps], sb[kOzMaxSteps], sacc[kOzMaxSteps];
    unsigned sfree[kOzMaxSteps];
  };
  int ngroups;
  Grp g[2];
  // The last group takes the top four diagonals (they need every slice of
  // A and B anyway); the first group the rest.  For s = 6 that is {0, 1}
  // (4 tile loads, 3 products) and {2..5} (12 loads, 18 products) per K
  // block.
  constexpr OzFixedSched() : ngroups(S > 4 ? 2 : 1), g{} {
    const int split = S > 4 ? S - 4 : 0;
    for (int gi = 0; gi < ngroups; ++gi) {
      Grp &G = g[gi];
      G.t0 = gi == 0 ? 0 : split;
      G.t1 = (ngroups == 1 || gi == 1) ? S - 1 : split - 1;
      int idxA[16] = {}, idxB[16] = {}, last[kOzMaxLoads] = {};
      for (int x = 0; x < 16; ++x) idxA[x] = idxB[x] = -1;
      for (int l = 0; l < kOzMaxLoads; ++l) G.first_use[l] = -1;
      const int pmax = G.t1 < S - 1 ? G.t1 : S - 1;
      for (int p = 0; p <= pmax; ++p) {
        const int qlo = G.t0 - p > 0 ? G.t0 - p : 0;
        const int qhi = G.t1 - p < S - 1 ? G.t1 - p : S - 1;
        if (qlo > qhi) continue;
        for (int q = qhi; q >= qlo; --q)
          if (idxB[q] < 0) {
            idxB[q] = G.nloads;
            G.side[G.nloads] = 1;
            G.slice[G.nloads++] = q;
          }
        idxA[p] = G.nloads;
        G.side[G.nloads] = 0;
        G.slice[G.nloads++] = p;
        for (int q = qlo; q <= qhi; ++q) {
          const int st = G.nsteps++;
          G.sa[st] = idxA[p];
          G.sb[st] = idxB[q];
          G.sacc[st] = p + q - G.t0;
          if (G.first_use[idxA[p]] < 0) G.first_use[idxA[p]] = st;
          if (G.first_use[idxB[q]] < 0) G.first_use[idxB[q]] = st;
          last[idxA[p]] = st;
          last[idxB[q]] = st;
        }
      }
      for (int l = 0; l < G.nloads; ++l) G.sfree[last[l]] |= 1u << l;
    }
  }
};

// Tile t of a problem -> (mt, nt), in bands of `band` m-tiles: within a
// band the n-tiles advance slowest, so the CTAs of one wave share a few A
// panels and a band's worth of B panels instead of every B panel.
__device__ __forceinline__ void tile_coords(int t, int mtiles, int ntiles, int band_m, int &mt, int &nt) {
  const int per_band = band_m * ntiles;
  const int band = t / per_band, r = t - band * per_band;
  const int m0 = band * band_m;
  const int bm = mtiles - m0 < band_m ? mtiles - m0 : band_m;
  mt = m0 + r % bm;
  nt = r / bm;
}

// m-tiles per raster band of the Ozaki GEMMs (bands of 4 to 64 m-tiles,
// and evict-first C traffic, measured the same on the 4096 x 4096 x 2304
// permuted contraction: 0.739-0.741 ms per GEMM launch).
constexpr int kOzBandM = 16;

// Ring slot and phase parity of load l of a block whose first load has
// global index L (l < 2 * kOzSlots).
__device__ __forceinline__ void oz_slot(uint32_t s0, uint32_t par0, int l, uint32_t &slot,
                                        uint32_t &par) {
  const uint32_t idx = s0 + (uint32_t)l;
  const uint32_t w = (idx >= kOzSlots ? 1u : 0u) + (idx >= 2 * kOzSlots ? 1u : 0u);
  slot = idx - w * kOzSlots;
  par = par0 ^ (w & 1u);
}

#include "oz_fixed.cuh"
#include "oz_2sm.cuh"

// The group schedule of the v2 kernel for s slices (host).
static OzSched build_oz_sched(int s) {
  OzSched S;
  std::memset(&S, 0, sizeof(S));
  S.ngroups = s > 4 ? 2 : 1;
  for (int gi = 0; gi < S.ngroups; ++gi) {
    OzGroup &G = S.g[gi];
    G.t0 = gi == 0 ? 0 : 4;
    G.t1 = gi == 0 ? std::min(3, s - 1) : std::min(7, s - 1);
    int idxA[16], idxB[16];
    for (int x = 0; x < 16; ++x) idxA[x] = idxB[x] = -1;
    int last[kOzMaxLoads];
    for (int p = 0; p <= std::min(G.t1, s - 1); ++p) {
      const int qlo = std::max(0, G.t0 - p), qhi = std::min(G.t1 - p, s - 1);
      if (qlo > qhi) continue;
      for (int q = qhi; q >= qlo; --q)
        if (idxB[q] < 0) {
          idxB[q] = G.nloads;
          G.load_side[G.nloads] = 1;
          G.load_slice[G.nloads++] = (int8_t)q;
        }
      idxA[p] = G.nloads;
      G.load_side[G.nloads] = 0;
      G.load_slice[G.nloads++] = (int8_t)p;
      for (int q = qlo; q <= qhi; ++q) {
        G.step_a[G.nsteps] = (int8_t)idxA[p];
        G.step_b[G.nsteps] = (int8_t)idxB[q];
        G.step_acc[G.nsteps] = (int8_t)(p + q - G.t0);
        last[idxA[p]] = G.nsteps;
        last[idxB[q]] = G.nsteps;
        ++G.nsteps;
      }
    }
    for (int l = 0; l < G.nloads; ++l) G.step_free[last[l]] |= (uint16_t)(1u << l);
  }
  return S;
}

// Non-finite rows of A / columns of B (flagged by the pack): those elements
// of C are computed here directly in FP64 (IEEE semantics), and the GEMM's
// epilogue skipped them.
// T is double or cplx<double>.  The flagged lists hold real (virtual) rows
// of the A and B panels: in the 1m layout (layout 1) rows 2i and 2i+1 of A
// are both flagged and the even one stands for complex row i; in the planar
// layout (2) the same holds for the rows of B (columns of C).
template <class T>
__device__ __forceinline__ void oz_fixup_range(const Operands &op, const Scalars<T> &s, int layout,
                                               const int32_t *rows, const int32_t *nrows,
                                               const int32_t *cols, const int32_t *ncols,
                                               const int32_t *expA, int64_t first, int64_t stride) {
  const int nr = *nrows, nc = *ncols;
  const int64_t total = (int64_t)nr * op.N + (int64_t)nc * op.M;
  for (int64_t e = first; e < total; e += stride) {
    int64_t i, j;
    if (e < (int64_t)nr * op.N) {
      i = rows[e / op.N];
      j = e % op.N;
      if (layout == 1) {
        if (i & 1) continue;
        i >>= 1;
      }
    } else {
      int64_t f = e - (int64_t)nr * op.N;
      j = cols[f / op.M];
      i = f % op.M;
      if (layout == 2) {
        if (j & 1) continue;
        j >>= 1;
      }
      if (expA[layout == 1 ? 2 * i : i] == kNonFinite) continue;  // done by the row pass
    }
    T acc = tzero<T>();
    for (int64_t k = 0; k < op.K; ++k) {
      T x = Loader<T>::load(op.A, op.Abase + op.offMA[i] + op.offKA[k], op.TA, op.conjA);
      T y = Loader<T>::load(op.B, op.Bbase + op.offNB[j] + op.offKB[k], op.TB, op.conjB);
      acc = cfma(x, y, acc);
    }
    const int64_t idx = op.Cbase + op.offMC[i] + op.offNC[j];
    const T old = s.beta_case == 0 ? tzero<T>() : load_c<T>(op.C, idx, op.TC);
    store_c<T>(op.C, idx, op.TC, axpby(s, acc, old));
  }
}

// The fixup of one plan: its operands, scalars and non-finite lists.
struct FixupJob {
  Operands op;
  double alpha[2], beta[2];
  int beta_case, cplx;
  const int32_t *rows, *nrows, *cols, *ncols, *expA;
};

__device__ __forceinline__ void oz_fixup_job(const FixupJob &f, int64_t first, int64_t stride) {
  if (f.cplx) {
    Scalars<cplx<double>> s;
    s.alpha.re = f.alpha[0]; s.alpha.im = f.alpha[1];
    s.beta.re = f.beta[0]; s.beta.im = f.beta[1];
    s.beta_case = f.beta_case;
    oz_fixup_range<cplx<double>>(f.op, s, f.cplx, f.rows, f.nrows, f.cols, f.ncols, f.expA, first, stride);
  } else {
    Scalars<double> s;
    s.alpha = f.alpha[0];
    s.beta = f.beta[0];
    s.beta_case = f.beta_case;
    oz_fixup_range<double>(f.op, s, 0, f.rows, f.nrows, f.cols, f.ncols, f.expA, first, stride);
  }
}

__global__ void __launch_bounds__(256) oz_fixup_kernel(const __grid_constant__ FixupJob f) {
  oz_fixup_job(f, blockIdx.x * (int64_t)blockDim.x + threadIdx.x, (int64_t)gridDim.x * blockDim.x);
}

// ------------------------------------------------------------- host side ---

static int64_t cdiv(int64_t a, int64_t b) { return (a + b - 1) / b; }

int tc_auto_method(const qs_plan *p) {
  // The tensor-core paths pay a pack pass, five more launches and pad to
  // 128 x 128 tiles: worth it once M fills a tile, N at least half of one,
  // K one K block, and the work is past the point where launch latency
  // dominates (M*N*K >= 2^26).  Complex plans count their real GEMM
  // (2 real rows or columns per complex one).
  const int64_t m = is_complex(p->T) ? 2 * p->M : p->M;
  const int64_t n = is_complex(p->T) ? 2 * p->N : p->N;
  if (m < 128 || n < 64 || p->K < 64) return QS_METHOD_NATIVE;
  if ((double)p->M * (double)p->N * (double)p->K < 67108864.0) return QS_METHOD_NATIVE;
  // Single precision too: 4 INT8 digits (10 products) stay within 1e-5 of
  // FP64 (about 1e-9 before the final rounding), where split BF16x3 keeps
  // about 16 mantissa bits (~1e-5 relative error on its own); BF16x3 stays
  // available by request.
  return QS_METHOD_OZAKI_I8;
}

// Slice counts with a compile-time (fixed-schedule) GEMM kernel.
static bool oz_fixed_slices(int s) { return s == 4 || s == 6 || s == 7; }

static int default_slices(int64_t K, bool cplx, bool dbl) {
  // The relative error of s base-256 digits is about 256^-s times
  // (row max / row rms of A + column max / column rms of B): ~1e-14 for
  // s = 6 on uniform inputs at K = 2304 (max/rms = sqrt 3), but up to ~1e-13
  // for Gaussian rows of a few thousand elements (max/rms ~ 4), which the
  // 1m form of complex data (K doubled) reaches.  7 digits (28 products)
  // for complex compute types and for K beyond 4096, else 6 (21 products).
  // Single precision (24 significand bits) needs 4 digits: ~1e-9 relative
  // before the one rounding to Float32.
  if (!dbl) return 4;
  int s = 6;
  if (cplx || K > 4096) s = 7;
  return s;
}

void tc_geometry(qs_plan *p) {
  TensorCoreGeom &g = p->tc;
  g = TensorCoreGeom{};
  // Complex plans run as one real GEMM with K doubled.  1m: A as "1e"
  // (2M rows), B as "1r"; planar: A as "1r", B as "1e" (2N columns), so C's
  // Re/Im sit in adjacent columns.  The expanded operand's panels are twice
  // the other's, so by default the smaller side is expanded (planar when
  // M > N); complex_mode forces one.
  const bool cx = is_complex(p->T);
  int layout = 0;
  if (cx) {
    if (p->opts.complex_mode == QS_CPLX_PLANAR) layout = 2;
    else if (p->opts.complex_mode == QS_CPLX_1M) layout = 1;
    else layout = p->M > p->N ? 2 : 1;
  }
  g.cplx_layout = layout;
  p->complex_mode = layout == 2 ? QS_CPLX_PLANAR : (layout == 1 ? QS_CPLX_1M : QS_CPLX_NONE);
  g.rows_per_elem_a = layout == 1 ? 2 : 1;
  g.cols_per_elem_b = layout == 2 ? 2 : 1;
  g.kmul = cx ? 2 : 1;
  const int64_t Mv = p->M * g.rows_per_elem_a, Nv = p->N * g.cols_per_elem_b;
  const int64_t Kv = cx ? 2 * p->K : p->K;
  if (p->method == QS_METHOD_OZAKI_I8) {
    g.nslices = p->opts.ozaki_slices > 0 ? p->opts.ozaki_slices : default_slices(Kv, cx, is_double(p->T));
    p->ozaki_slices = g.nslices;
    g.kblocks = cdiv(Kv, 128);
    g.mtiles = cdiv(Mv, 128);
    g.ntiles = cdiv(Nv, 128);
    // The CTA-pair kernel (6 or 7 slices) reads M tiles in pairs: the A
    // panel holds an even number of them (a padding tile's rows are never
    // stored, and rows of A do not mix).
    const int64_t mt_alloc = oz_fixed_slices(g.nslices) ? (g.mtiles + 1) / 2 * 2 : g.mtiles;
    g.Mp = mt_alloc * 128;
    g.Np = g.ntiles * 128;
    g.plane_bytes_a = mt_alloc * g.kblocks * 128 * 128;
    g.plane_bytes_b = g.ntiles * g.kblocks * 128 * 128;
    // INT32-exact segment: (terms) * kblocks * 128 * 128^2 < 2^31 (digits
    // in [-128, 127]).
    int64_t maxkb = (int64_t)(2147483647ll / ((int64_t)g.nslices * 128 * 128 * 128));
    if (maxkb < 1) maxkb = 1;
    g.kseg = (int)std::min<int64_t>(maxkb, g.kblocks);
  } else {
    g.nslices = 2;
    g.kblocks = cdiv(Kv, 64);
    g.mtiles = cdiv(Mv, 128);
    g.ntiles = cdiv(Nv, 128);
    g.Mp = g.mtiles * 128;
    g.Np = g.ntiles * 128;
    g.plane_bytes_a = g.mtiles * g.kblocks * 128 * 128;
    g.plane_bytes_b = g.ntiles * g.kblocks * 128 * 128;
    g.kseg = (int)std::min<int64_t>(kBf16SegK / 64, g.kblocks);
  }
}

static int tc_alloc(qs_plan *p, void **out, size_t bytes) { return plan_alloc(p, out, bytes); }

// Tensor maps of the packed Ozaki panels for the CTA-pair kernel: each panel
// as a 2-D array of 128-byte rows (slices x tiles x K blocks x 128 rows),
// copied unswizzled (the tiles are stored swizzled); boxes of 128 rows for A
// and 64 rows (one CTA's half of a B tile) for B.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    cudaGetLastError();
  }
  return fn;
}

static bool encode_panel_map(CUtensorMap *m, void *base, uint64_t rows, uint32_t box_rows) {
  auto enc = tensor_map_encoder();
  if (!enc || rows == 0 || rows > 0x7fffffffull || (reinterpret_cast<uintptr_t>(base) & 15)) return false;
  const cuuint64_t dims[2] = {128, rows};
  const cuuint64_t strides[1] = {128};
  const cuuint32_t box[2] = {128, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

static bool make_pair_maps(qs_plan *p) {
  static_assert(sizeof(CUtensorMap) == 128, "tensor map size");
  const TensorCoreGeom &g = p->tc;
  CUtensorMap ma, mb;
  if (!encode_panel_map(&ma, p->ws.panelA, (uint64_t)g.plane_bytes_a * g.nslices / 128, 128) ||
      !encode_panel_map(&mb, p->ws.panelB, (uint64_t)g.plane_bytes_b * g.nslices / 128, 64))
    return false;
  std::memcpy(p->oz_tmap, &ma, 128);
  std::memcpy(p->oz_tmap + 128, &mb, 128);
  return true;
}

// The pack's row order for a real operand (side 0: A over M, 1: B over N)
// whose unit-stride axis is neither the first label of its row group nor
// the first K label but a later row label d*: rows enumerated with d*
// fastest, then the others in order (row index r = sum_d x_d R_d, first
// label fastest).  Padding rows keep their place.  Else no table.
static int upload_row_order(qs_plan *p, int side) {
  const TensorCoreGeom &g = p->tc;
  const Group &G = side == 0 ? p->mg : p->ng;
  const int T = side == 0 ? p->TA : p->TB;
  if (g.cplx_layout != 0 || is_complex(T) || G.D < 2) return QS_OK;
  auto unit = [](int64_t st, int64_t len) { return len > 1 && (st == 1 || st == -1); };
  if (unit(G.st[0][0], G.len[0])) return QS_OK;                        // rows already unit-stride
  if (p->kg.D > 0 && unit(p->kg.st[side][0], p->kg.len[0])) return QS_OK;  // K-fast gather
  int ds = -1;
  for (int d = 1; d < G.D && ds < 0; ++d)
    if (unit(G.st[0][d], G.len[d])) ds = d;
  if (ds < 0) return QS_OK;
  const int64_t rows = G.length(), rows_pad = side == 0 ? g.Mp : g.Np;
  if (rows <= 0 || rows_pad > INT32_MAX) return QS_OK;
  int64_t R[kMaxRank];
  int64_t acc = 1;
  for (int d = 0; d < G.D; ++d) {
    R[d] = acc;
    acc *= G.len[d];
  }
  int order[kMaxRank], n = 0;
  order[n++] = ds;
  for (int d = 0; d < G.D; ++d)
    if (d != ds) order[n++] = d;
  std::vector<int32_t> h((size_t)rows_pad);
  int64_t x[kMaxRank] = {};
  for (int64_t i = 0; i < rows; ++i) {
    int64_t r = 0;
    for (int d = 0; d < G.D; ++d) r += x[d] * R[d];
    h[(size_t)i] = (int32_t)r;
    for (int q = 0; q < n; ++q) {  // next coordinate, order[0] fastest
      const int d = order[q];
      if (++x[d] < G.len[d]) break;
      x[d] = 0;
    }
  }
  for (int64_t i = rows; i < rows_pad; ++i) h[(size_t)i] = (int32_t)i;
  void *q;
  int rc = tc_alloc(p, &q, h.size() * sizeof(int32_t));
  if (rc) return rc;
  if (setup_upload(q, h.data(), h.size() * sizeof(int32_t)) != cudaSuccess)
    return fail(QS_ECUDA, "cudaMemcpyAsync (pack row order)");
  p->ws.rperm[side] = (int32_t *)q;
  return QS_OK;
}

int tc_prepare(qs_plan *p) {
  tc_geometry(p);
  const TensorCoreGeom &g = p->tc;
  int rc;
  void *q;
  if ((rc = tc_alloc(p, &q, (size_t)g.plane_bytes_a * g.nslices))) return rc;
  p->ws.panelA = q;
  if ((rc = tc_alloc(p, &q, (size_t)g.plane_bytes_b * g.nslices))) return rc;
  p->ws.panelB = q;
  if (p->method == QS_METHOD_OZAKI_I8) {
    if ((rc = tc_alloc(p, &q, (size_t)(g.Mp + g.Np) * sizeof(unsigned long long)))) return rc;
    p->ws.rowmax = (unsigned long long *)q;
    for (int side = 0; side < 2; ++side)
      if ((rc = upload_row_order(p, side))) return rc;
  }
  if (p->method == QS_METHOD_OZAKI_I8 && oz_fixed_slices(g.nslices) &&
      !(p->opts.flags & (QS_PLAN_OZ_SINGLE_SM | QS_PLAN_PER_PRODUCT_GEMM)))
    p->oz_pair_maps = make_pair_maps(p) ? 1 : 0;  // else the one-SM kernel runs
  if (p->method == QS_METHOD_OZAKI_I8) {
    // exponents (padded rows/cols), non-finite lists, their counters, status
    size_t n = (size_t)(g.Mp + g.Np + g.Mp + g.Np + 4);
    if ((rc = tc_alloc(p, &q, n * sizeof(int32_t)))) return rc;
    int32_t *b = (int32_t *)q;
    p->ws.expA = b;
    p->ws.expB = b + g.Mp;
    if (setup_zero_async(q, n * sizeof(int32_t)) != cudaSuccess) return fail(QS_ECUDA, "cudaMemsetAsync");
    p->ws.status = b + n - 1;
  } else {
    if ((rc = tc_alloc(p, &q, 4 * sizeof(int32_t)))) return rc;
    if (setup_zero_async(q, 4 * sizeof(int32_t)) != cudaSuccess) return fail(QS_ECUDA, "cudaMemsetAsync");
    p->ws.status = (int32_t *)q;
  }
  static bool attr_set[2] = {false, false};
  if (!attr_set[0]) {
    cudaFuncSetAttribute(tc_gemm_kernel<KIND_I8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)gemm_smem_bytes<KIND_I8>());
    cudaFuncSetAttribute(tc_gemm_kernel<KIND_BF16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)gemm_smem_bytes<KIND_BF16>());
    cudaFuncSetAttribute(oz_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)oz_smem_bytes());
    cudaFuncSetAttribute(oz_gemm_fixed_kernel<6, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)oz_smem_bytes());
    cudaFuncSetAttribute(oz_gemm_fixed_kernel<7, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)oz_smem_bytes());
    cudaFuncSetAttribute(oz_gemm_fixed_kernel<6, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)oz_smem_bytes());
    cudaFuncSetAttribute(oz_gemm_fixed_kernel<7, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)oz_smem_bytes());
    cudaFuncSetAttribute(oz_gemm_fixed_kernel<4, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)oz_smem_bytes());
    cudaFuncSetAttribute(oz_gemm_pair_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)oz_smem_bytes());
    cudaFuncSetAttribute(oz_gemm_fixed_kernel<4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)oz_smem_bytes());
    cudaFuncSetAttribute(oz_gemm_pair_kernel<6>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)oz_smem_bytes());
    cudaFuncSetAttribute(oz_gemm_pair_kernel<7>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)oz_smem_bytes());
    attr_set[0] = attr_set[1] = true;
  }
  return QS_OK;
}

static int num_sms() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return sms;
}

static PackArgs pack_args(const qs_plan *p, int side) {
  const TensorCoreGeom &g = p->tc;
  PackArgs a;
  if (side == 0) {
    a.X = p->Adata; a.Xbase = p->Abase; a.TX = p->TA; a.conj = p->conjA;
    a.offR = p->ws.offM[0]; a.offK = p->ws.offK[0];
    a.rows = p->M * g.rows_per_elem_a; a.rows_pad = g.Mp; a.tile_rows = 128;
    a.cmode = g.cplx_layout == 1 ? 1 : (g.cplx_layout == 2 ? 2 : 0);
    a.rfast = p->a_mfast;
    a.panel = (uint8_t *)p->ws.panelA; a.plane = g.plane_bytes_a;
    a.exp_out = p->ws.expA;
  } else {
    a.X = p->Bdata; a.Xbase = p->Bbase; a.TX = p->TB; a.conj = p->conjB;
    a.offR = p->ws.offN[0]; a.offK = p->ws.offK[1];
    a.rows = p->N * g.cols_per_elem_b; a.rows_pad = g.Np;
    a.tile_rows = 128;
    a.cmode = g.cplx_layout == 1 ? 2 : (g.cplx_layout == 2 ? 1 : 0);
    a.rfast = p->b_nfast;
    a.panel = (uint8_t *)p->ws.panelB; a.plane = g.plane_bytes_b;
    a.exp_out = p->ws.expB;
  }
  a.K = p->K * g.kmul;
  a.kblocks = (int)g.kblocks;
  a.nslices = g.nslices;
  a.rowmax = p->ws.rowmax ? p->ws.rowmax + (side == 0 ? 0 : g.Mp) : nullptr;
  a.rperm = p->ws.rperm[side];
  if (a.rperm) a.rfast = 1;
  if (p->method == QS_METHOD_OZAKI_I8) {
    int32_t *lists = p->ws.expA + g.Mp + g.Np;  // [rows: Mp][cols: Np][2 counters]
    int32_t *counters = lists + g.Mp + g.Np;
    a.flag_list = side == 0 ? lists : lists + g.Mp;
    a.flag_count = counters + side;
  } else {
    a.flag_list = a.flag_count = nullptr;
    a.exp_out = nullptr;
  }
  return a;
}

static GemmArgs make_gemm_args(const qs_plan *p, const double *alpha, const double *beta,
                               int beta_case) {
  const TensorCoreGeom &g = p->tc;
  const bool oz = p->method == QS_METHOD_OZAKI_I8;
  GemmArgs a;
  a.panelA = (const uint8_t *)p->ws.panelA;
  a.panelB = (const uint8_t *)p->ws.panelB;
  a.planeA = g.plane_bytes_a;
  a.planeB = g.plane_bytes_b;
  a.mtiles = (int)g.mtiles;
  a.ntiles = (int)g.ntiles;
  a.kblocks = (int)g.kblocks;
  a.nslices = g.nslices;
  a.kseg_blocks = g.kseg;
  a.nkseg = (int)cdiv(g.kblocks, g.kseg);
  a.expA = p->ws.expA;
  a.expB = p->ws.expB;
  a.C = p->Cdata;
  a.Cbase = p->Cbase;
  a.TC = p->TC;
  a.offMC = p->ws.offM[1];
  a.offNC = p->ws.offN[1];
  a.M = p->M * g.rows_per_elem_a;
  a.N = p->N * g.cols_per_elem_b;
  a.cplx = g.cplx_layout;
  // alpha/beta converted to the compute type first (convert(T, alpha)); the
  // Ozaki epilogue then works in FP64 and rounds once to eltype(C).
  auto cv = [p](double x) { return is_double(p->T) ? x : (double)(float)x; };
  a.alpha_im = cv(alpha[1]);
  a.beta_im = cv(beta[1]);
  a.alpha = cv(alpha[0]);
  a.beta = cv(beta[0]);
  a.beta_case = beta_case;
  a.status = p->ws.status;
  // Diagonal t holds products of digits p + q = t + 2 (weight 256^-(t+2)),
  // times (128/127)^2 for the two operands' digit scale.
  const double undo = (128.0 / 127.0) * (128.0 / 127.0);
  for (int t = 0; t < 16; ++t) a.wdiag[t] = std::ldexp(undo, -8 * (t + 2));
  a.wait_ns = p->wait_ns;
  a.hold_loads = p->hold_loads;
  a.band_m = kOzBandM;
  return a;
}

static FixupJob make_fixup_job(const qs_plan *p, const double *alpha, const double *beta,
                               int beta_case) {
  const TensorCoreGeom &g = p->tc;
  FixupJob f;
  Operands &op = f.op;
  op.A = p->Adata; op.B = p->Bdata; op.C = p->Cdata;
  op.Abase = p->Abase; op.Bbase = p->Bbase; op.Cbase = p->Cbase;
  op.TA = p->TA; op.TB = p->TB; op.TC = p->TC;
  op.conjA = p->conjA; op.conjB = p->conjB;
  op.offMA = p->ws.offM[0]; op.offMC = p->ws.offM[1];
  op.offNB = p->ws.offN[0]; op.offNC = p->ws.offN[1];
  op.offKA = p->ws.offK[0]; op.offKB = p->ws.offK[1];
  op.M = p->M; op.N = p->N; op.K = p->K;
  auto cv = [p](double x) { return is_double(p->T) ? x : (double)(float)x; };
  f.alpha[0] = cv(alpha[0]); f.alpha[1] = cv(alpha[1]);
  f.beta[0] = cv(beta[0]); f.beta[1] = cv(beta[1]);
  f.beta_case = beta_case;
  f.cplx = g.cplx_layout;
  int32_t *lists = p->ws.expA + g.Mp + g.Np;  // [rows: Mp][cols: Np][2 counters]
  int32_t *counters = lists + g.Mp + g.Np;
  f.rows = lists;
  f.nrows = counters;
  f.cols = lists + g.Mp;
  f.ncols = counters + 1;
  f.expA = p->ws.expA;
  return f;
}

// The CTA-pair Ozaki GEMM: clusters of two CTAs, as many as fit at once
// (persistent), each pair looping over 256 x 128 tiles of C.
static cudaError_t launch_oz_pair(int S, const GemmArgs &a, const unsigned char *maps, cudaStream_t st) {
  CUtensorMap ma, mb;
  std::memcpy(&ma, maps, 128);
  std::memcpy(&mb, maps + 128, 128);
  static int max_clusters[3] = {0, 0, 0};
  const int si = S == 4 ? 0 : S == 6 ? 1 : 2;
  const void *kern = S == 4 ? (const void *)oz_gemm_pair_kernel<4>
                   : S == 6 ? (const void *)oz_gemm_pair_kernel<6> : (const void *)oz_gemm_pair_kernel<7>;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(320, 1, 1);
  cfg.dynamicSmemBytes = oz_smem_bytes();
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (!max_clusters[si]) {
    cfg.gridDim = dim3(2 * (unsigned)(num_sms() / 2), 1, 1);
    int n = 0;
    cudaError_t e = cudaOccupancyMaxActiveClusters(&n, kern, &cfg);
    if (e != cudaSuccess || n < 1) {
      cudaGetLastError();
      return e != cudaSuccess ? e : cudaErrorInvalidConfiguration;
    }
    max_clusters[si] = n;
  }
  const int pairs = (a.mtiles + 1) / 2 * a.ntiles;
  const int clusters = std::min(pairs, max_clusters[si]);
  cfg.gridDim = dim3(2 * (unsigned)clusters, 1, 1);
  if (S == 4) return cudaLaunchKernelEx(&cfg, oz_gemm_pair_kernel<4>, a, ma, mb);
  if (S == 6) return cudaLaunchKernelEx(&cfg, oz_gemm_pair_kernel<6>, a, ma, mb);
  return cudaLaunchKernelEx(&cfg, oz_gemm_pair_kernel<7>, a, ma, mb);
}

int tc_execute(qs_plan *p, const double *alpha, const double *beta, int beta_case,
               cudaStream_t st, cudaEvent_t *ev) {
  const TensorCoreGeom &g = p->tc;
  const bool oz = p->method == QS_METHOD_OZAKI_I8;
  int launches = 0;
  cudaError_t e;
  if (oz) {
    int32_t *counters = p->ws.expA + g.Mp + g.Np + g.Mp + g.Np;
    e = cudaMemsetAsync(counters, 0, 2 * sizeof(int32_t), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(p->ws.rowmax, 0, (size_t)(g.Mp + g.Np) * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return fail(QS_ECUDA, "cudaMemsetAsync");
  }
  if (ev) cudaEventRecord(ev[0], st);
  {
    // Profile stages: Ozaki: ev[1] after A's two passes, ev[2] after B's;
    // BF16x3 (both operands per launch): both after the pack.
    const PackArgs pa = pack_args(p, 0), pb = pack_args(p, 1);
    const int nrbA = (int)cdiv(pa.rows_pad, 32), nrbB = (int)cdiv(pb.rows_pad, 32);
    const int64_t nA = (int64_t)nrbA * g.kblocks, nB = (int64_t)nrbB * g.kblocks;
    if (oz) {
      launch_pack_operand(pa, st);
      if (ev) cudaEventRecord(ev[1], st);
      launch_pack_operand(pb, st);
      if (ev) cudaEventRecord(ev[2], st);
      launches += 4;
    } else {
      bf16_pack_pair_kernel<<<(unsigned)(nA + nB), 256, 0, st>>>(pa, pb, nrbA, nrbB, nA);
      if (ev) {
        cudaEventRecord(ev[1], st);
        cudaEventRecord(ev[2], st);
      }
      ++launches;
    }
  }
  const GemmArgs a = make_gemm_args(p, alpha, beta, beta_case);
  const int tiles = a.mtiles * a.ntiles;
  const int grid = std::min(tiles, num_sms());
  if (oz) {
    if (p->opts.flags & QS_PLAN_PER_PRODUCT_GEMM) {
      tc_gemm_kernel<KIND_I8><<<grid, 192, gemm_smem_bytes<KIND_I8>(), st>>>(a, GemmTable{nullptr, nullptr, nullptr, 0});
    } else if (oz_fixed_slices(g.nslices) && p->oz_pair_maps) {
      e = launch_oz_pair(g.nslices, a, p->oz_tmap, st);
      if (e != cudaSuccess) return fail(QS_ECUDA, std::string("CTA-pair GEMM launch: ") + cudaGetErrorString(e));
    } else if (g.nslices == 4) {
      oz_gemm_fixed_kernel<4, false><<<grid, 320, oz_smem_bytes(), st>>>(a, GemmTable{nullptr, nullptr, nullptr, 0});
    } else if (g.nslices == 6) {
      oz_gemm_fixed_kernel<6, false><<<grid, 320, oz_smem_bytes(), st>>>(a, GemmTable{nullptr, nullptr, nullptr, 0});
    } else if (g.nslices == 7) {
      oz_gemm_fixed_kernel<7, false><<<grid, 320, oz_smem_bytes(), st>>>(a, GemmTable{nullptr, nullptr, nullptr, 0});
    } else if (g.nslices <= 8) {
      const OzSched sched = build_oz_sched(g.nslices);
      oz_gemm_kernel<<<grid, 320, oz_smem_bytes(), st>>>(a, sched);
    } else {
      tc_gemm_kernel<KIND_I8><<<grid, 192, gemm_smem_bytes<KIND_I8>(), st>>>(a, GemmTable{nullptr, nullptr, nullptr, 0});
    }
  } else {
    tc_gemm_kernel<KIND_BF16><<<grid, 192, gemm_smem_bytes<KIND_BF16>(), st>>>(a, GemmTable{nullptr, nullptr, nullptr, 0});
  }
  ++launches;
  if (ev) cudaEventRecord(ev[3], st);
  if (oz) {
    const FixupJob f = make_fixup_job(p, alpha, beta, beta_case);
    oz_fixup_kernel<<<64, 256, 0, st>>>(f);
    ++launches;
    if (ev) cudaEventRecord(ev[4], st);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    std::ostringstream s;
    s << "CUDA error in tensor-core launch: " << cudaGetErrorString(e);
    return fail(QS_ECUDA, s.str());
  }
  count_launches(launches);
  p->prof_nstages = oz ? 4 : 3;
  return QS_OK;
}

// ---------------------------------------------------------- grouped ---
// Many independent plans of one class as one launch per stage: pack (fused
// row-max and digit planes, or the BF16 planes), the persistent GEMM over a problem table,
// and the non-finite fixup.  Each plan keeps its own workspace; the launch
// reads per-problem arguments from device tables.

// One operand side of one problem in a grouped pack launch: blocks
// [block_start, block_start + gx * kblocks) of the launch, gx row blocks of
// 32 rows by kblocks K blocks (Ozaki: 128 K values; BF16x3: 64).
struct PackJob {
  PackArgs pa;
  int gx;
  int block_start;
};

// A per-plan prep: the non-finite counters and the row maxima to zero.
struct ZeroJob {
  int32_t *counters;
  unsigned long long *rowmax;
  int64_t nrows;
};

// One block per plan (grid-strided).
__global__ void __launch_bounds__(256) oz_prep_grouped(const ZeroJob *jobs, int n) {
  for (int j = blockIdx.x; j < n; j += gridDim.x) {
    const ZeroJob z = jobs[j];
    if (threadIdx.x < 2) z.counters[threadIdx.x] = 0;
    for (int64_t i = threadIdx.x; i < z.nrows; i += blockDim.x) z.rowmax[i] = 0;
  }
}

// The two pack passes over a chunk of (problem, side) jobs: job j owns
// blocks [block_start, block_start + gx * kblocks) of the group (row block
// fastest), jobmap[b] the job of block b, and a launch covers the chunk's
// blocks from b0; pass 1 skips the K blocks past K.  A group packs chunk by
// chunk (pass 1, pass 2, next chunk), each chunk's operands small enough
// that pass 2 re-reads them from L2.
// The block's job in shared memory (one coalesced load of the whole record,
// so the pass reads its arguments from shared memory instead of a chain of
// dependent loads from the job table), and the block's (r0, k0).
__device__ __forceinline__ void stage_pack_job(const PackJob *jobs, const int *jobmap, int b, PackJob &sj,
                                               int64_t &r0, int64_t &k0) {
  static_assert(sizeof(PackJob) % 8 == 0, "PackJob copies as 8-byte words");
  const uint64_t *src = reinterpret_cast<const uint64_t *>(jobs + __ldg(jobmap + b));
  if (threadIdx.x < sizeof(PackJob) / 8) reinterpret_cast<uint64_t *>(&sj)[threadIdx.x] = __ldg(src + threadIdx.x);
  __syncthreads();
  const int lb = b - sj.block_start;
  r0 = (int64_t)(lb % sj.gx) * kPackRows;
  k0 = (int64_t)(lb / sj.gx) * kPackK;
}

template <int KIND>
__global__ void __launch_bounds__(256, 6) oz_rowmax_grouped(const PackJob *jobs, const int *jobmap, int b0) {
  __shared__ PackJob sj;
  int64_t r0, k0;
  stage_pack_job(jobs, jobmap, b0 + (int)blockIdx.x, sj, r0, k0);
  if (k0 >= sj.pa.K) return;
  oz_rowmax_block<KIND, true>(sj.pa, r0, k0);
}

template <int KIND>
__global__ void __launch_bounds__(256, 4) oz_digit_grouped(const PackJob *jobs, const int *jobmap, int b0) {
  __shared__ PackJob sj;
  int64_t r0, k0;
  stage_pack_job(jobs, jobmap, b0 + (int)blockIdx.x, sj, r0, k0);
  oz_digit_block<KIND, true>(sj.pa, r0, k0);
}

__global__ void __launch_bounds__(256) bf16_pack_grouped(const PackJob *jobs, const int *jobmap) {
  const PackJob &j = jobs[__ldg(jobmap + blockIdx.x)];
  const int lb = blockIdx.x - j.block_start;
  const PackArgs pa = j.pa;
  bf16_pack_block(pa, (int64_t)(lb % j.gx) * 32, (int64_t)(lb / j.gx) * 64);
}

// One block per plan (grid-strided); a plan with nothing flagged returns at
// once.
__global__ void __launch_bounds__(256) oz_fixup_grouped(const FixupJob *jobs, int n) {
  for (int j = blockIdx.x; j < n; j += gridDim.x) {
    const FixupJob &f = jobs[j];
    if (*f.nrows == 0 && *f.ncols == 0) continue;
    oz_fixup_job(f, threadIdx.x, blockDim.x);
  }
}

int tc_group_class(const qs_plan *p) {
  if (p->method == QS_METHOD_BF16X3) return TC_CLASS_BF16;
  if (p->opts.flags & QS_PLAN_PER_PRODUCT_GEMM) return TC_CLASS_I8;
  if (p->tc.nslices == 4) return TC_CLASS_OZ4;
  if (p->tc.nslices == 6) return TC_CLASS_OZ6;
  if (p->tc.nslices == 7) return TC_CLASS_OZ7;
  return TC_CLASS_I8;
}

static size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

int tc_group_build(TcGroup &g, const double *alpha, const double *beta, const int *bcase) {
  const int n = (int)g.plans.size();
  const bool oz = g.cls != TC_CLASS_BF16;
  std::vector<PackJob> jobs;
  std::vector<GemmArgs> gemm;
  std::vector<int> tiles(1, 0);
  std::vector<ZeroJob> zero;
  std::vector<FixupJob> fix;
  int blocks = 0;
  for (int i = 0; i < n; ++i) {
    const qs_plan *p = g.plans[i];
    const TensorCoreGeom &tg = p->tc;
    const double *al = alpha + 2 * g.idx[i], *be = beta + 2 * g.idx[i];
    for (int side = 0; side < 2; ++side) {
      PackJob j;
      j.pa = pack_args(p, side);
      j.gx = (int)cdiv(j.pa.rows_pad, 32);
      j.block_start = blocks;
      const int64_t nb = (int64_t)j.gx * tg.kblocks;
      if (blocks + nb > INT_MAX) return fail(QS_EINVAL, "ArgumentError: grouped pack launch too large");
      blocks += (int)nb;
      jobs.push_back(j);
    }
    gemm.push_back(make_gemm_args(p, al, be, bcase[g.idx[i]]));
    const int64_t t = (int64_t)tiles.back() + (int64_t)tg.mtiles * tg.ntiles;
    if (t > INT_MAX) return fail(QS_EINVAL, "ArgumentError: grouped GEMM launch too large");
    tiles.push_back((int)t);
    if (oz) {
      ZeroJob z;
      z.counters = p->ws.expA + tg.Mp + tg.Np + tg.Mp + tg.Np;
      z.rowmax = p->ws.rowmax;
      z.nrows = tg.Mp + tg.Np;
      zero.push_back(z);
      fix.push_back(make_fixup_job(p, al, be, bcase[g.idx[i]]));
    }
  }
  g.njobs = (int)jobs.size();
  g.pack_blocks = blocks;
  // Pack chunks: consecutive jobs up to kPackChunkBytes of operand data
  // (a job larger than that is a chunk of its own).
  g.chunks.assign(1, 0);
  {
    size_t bytes = 0;
    for (size_t jj = 0; jj < jobs.size(); ++jj) {
      const PackArgs &pa = jobs[jj].pa;
      const size_t jb = (size_t)pa.rows * (size_t)pa.K * 8;  // about: 8 bytes per virtual element
      if (bytes > 0 && bytes + jb > kPackChunkBytes) {
        g.chunks.push_back(jobs[jj].block_start);
        bytes = 0;
      }
      bytes += jb;
    }
    if (blocks > 0) g.chunks.push_back(blocks);
    else g.chunks.clear();
  }
  std::vector<int> jobmap((size_t)blocks);
  for (size_t jj = 0; jj < jobs.size(); ++jj) {
    const int end = jj + 1 < jobs.size() ? jobs[jj + 1].block_start : blocks;
    std::fill(jobmap.begin() + jobs[jj].block_start, jobmap.begin() + end, (int)jj);
  }
  g.pack_kind = kPackAny;
  if (oz && !jobs.empty()) {
    g.pack_kind = pack_kind_of(jobs[0].pa);
    for (const PackJob &j : jobs)
      if (pack_kind_of(j.pa) != g.pack_kind) g.pack_kind = kPackAny;
  }
  g.tiles = tiles.back();
  std::vector<int> tilemap((size_t)g.tiles);
  for (int i = 0; i < n; ++i) std::fill(tilemap.begin() + tiles[i], tilemap.begin() + tiles[i + 1], i);
  size_t off = 0;
  g.off_pack = off;
  off = align_up(off + jobs.size() * sizeof(PackJob), 64);
  g.off_gemm = off;
  off = align_up(off + gemm.size() * sizeof(GemmArgs), 64);
  g.off_tiles = off;
  off = align_up(off + tiles.size() * sizeof(int), 64);
  g.off_zero = off;
  off = align_up(off + zero.size() * sizeof(ZeroJob), 64);
  g.off_fix = off;
  off = align_up(off + fix.size() * sizeof(FixupJob), 64);
  g.off_jobmap = off;
  off = align_up(off + jobmap.size() * sizeof(int), 64);
  g.off_tilemap = off;
  off = align_up(off + tilemap.size() * sizeof(int), 64);
  g.image.assign(off, 0);
  auto put = [&](size_t at, const void *src, size_t bytes) {
    if (bytes) std::memcpy(g.image.data() + at, src, bytes);
  };
  put(g.off_pack, jobs.data(), jobs.size() * sizeof(PackJob));
  put(g.off_gemm, gemm.data(), gemm.size() * sizeof(GemmArgs));
  put(g.off_tiles, tiles.data(), tiles.size() * sizeof(int));
  put(g.off_zero, zero.data(), zero.size() * sizeof(ZeroJob));
  put(g.off_fix, fix.data(), fix.size() * sizeof(FixupJob));
  put(g.off_jobmap, jobmap.data(), jobmap.size() * sizeof(int));
  put(g.off_tilemap, tilemap.data(), tilemap.size() * sizeof(int));
  return QS_OK;
}

// Stream-ordered: the tables are allocated on the build stream and freed on
// the group's release stream after their last use (tc_group_release), so
// building and dropping groups never synchronizes the device.
int tc_group_upload(TcGroup &g, cudaStream_t st) {
  if (g.dev) return fail(QS_EINVAL, "internal: grouped tables already uploaded");
  const int nchunks = (int)g.chunks.size() - 1;
  if (nchunks > 0) {
    cudaError_t e0 = cudaSuccess;
    if (!g.aux) e0 = cudaStreamCreateWithFlags(&g.aux, cudaStreamNonBlocking);
    while (e0 == cudaSuccess && (int)g.ev.size() < nchunks) {
      cudaEvent_t ev;
      e0 = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
      if (e0 == cudaSuccess) g.ev.push_back(ev);
    }
    if (e0 == cudaSuccess && !g.join) e0 = cudaEventCreateWithFlags(&g.join, cudaEventDisableTiming);
    if (e0 != cudaSuccess) return fail(QS_ECUDA, std::string("grouped pack streams: ") + cudaGetErrorString(e0));
  }
  cudaError_t e = cudaMallocAsync(&g.dev, g.image.size(), st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    g.dev = nullptr;
    return fail(QS_ENOMEM, "device allocation of a grouped launch's tables failed");
  }
  g.dev_bytes = g.image.size();
  e = cudaMemcpyAsync(g.dev, g.image.data(), g.image.size(), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return fail(QS_ECUDA, "cudaMemcpyAsync (grouped launch tables)");
  return QS_OK;
}

int tc_group_launch(const TcGroup &g, cudaStream_t st, int *launches) {
  const int n = (int)g.plans.size();
  if (n == 0) return QS_OK;
  uint8_t *d = (uint8_t *)g.dev;
  const PackJob *jobs = (const PackJob *)(d + g.off_pack);
  const GemmArgs *tab = (const GemmArgs *)(d + g.off_gemm);
  const int *tile_start = (const int *)(d + g.off_tiles);
  const GemmTable gt{tab, tile_start, (const int *)(d + g.off_tilemap), n};
  // The kernel's own GemmArgs: the first problem's (the launch-wide status
  // word and the table-independent fields).
  GemmArgs base;
  std::memcpy(&base, g.image.data() + g.off_gemm, sizeof(GemmArgs));
  const int grid = std::min(g.tiles, num_sms());
  int l = 0;
  if (g.cls == TC_CLASS_BF16) {
    bf16_pack_grouped<<<g.pack_blocks, 256, 0, st>>>(jobs, (const int *)(d + g.off_jobmap));
    tc_gemm_kernel<KIND_BF16><<<grid, 192, gemm_smem_bytes<KIND_BF16>(), st>>>(base, gt);
    l = 2;
  } else {
    const ZeroJob *zero = (const ZeroJob *)(d + g.off_zero);
    const FixupJob *fix = (const FixupJob *)(d + g.off_fix);
    const int pgrid = std::min(n, 4 * num_sms());
    oz_prep_grouped<<<(unsigned)std::min(n, 4 * num_sms()), 256, 0, st>>>(zero, n);
    const int *jobmap = (const int *)(d + g.off_jobmap);
    // Row maxima chunk by chunk on st; each chunk's digits on the aux stream
    // after it, so the row maxima of chunk c + 1 overlap the digits of c.
    const int nchunks = (int)g.chunks.size() - 1;
    if (nchunks > 0 && (!g.aux || (int)g.ev.size() < nchunks || !g.join))
      return fail(QS_EINVAL, "internal: grouped pack streams not created");
    for (int c = 0; c < nchunks; ++c) {
      const int b0 = g.chunks[c];
      const unsigned nb = (unsigned)(g.chunks[c + 1] - b0);
      switch (g.pack_kind) {
        case kPackF64: oz_rowmax_grouped<kPackF64><<<nb, 256, 0, st>>>(jobs, jobmap, b0); break;
        case kPackF32: oz_rowmax_grouped<kPackF32><<<nb, 256, 0, st>>>(jobs, jobmap, b0); break;
        default: oz_rowmax_grouped<kPackAny><<<nb, 256, 0, st>>>(jobs, jobmap, b0); break;
      }
      cudaEventRecord(g.ev[c], st);
      cudaStreamWaitEvent(g.aux, g.ev[c], 0);
      switch (g.pack_kind) {
        case kPackF64: oz_digit_grouped<kPackF64><<<nb, 256, 0, g.aux>>>(jobs, jobmap, b0); break;
        case kPackF32: oz_digit_grouped<kPackF32><<<nb, 256, 0, g.aux>>>(jobs, jobmap, b0); break;
        default: oz_digit_grouped<kPackAny><<<nb, 256, 0, g.aux>>>(jobs, jobmap, b0); break;
      }
    }
    if (nchunks > 0) {
      cudaEventRecord(g.join, g.aux);
      cudaStreamWaitEvent(st, g.join, 0);
    }
    if (g.cls == TC_CLASS_OZ4)
      oz_gemm_fixed_kernel<4, true><<<grid, 320, oz_smem_bytes(), st>>>(base, gt);
    else if (g.cls == TC_CLASS_OZ6)
      oz_gemm_fixed_kernel<6, true><<<grid, 320, oz_smem_bytes(), st>>>(base, gt);
    else if (g.cls == TC_CLASS_OZ7)
      oz_gemm_fixed_kernel<7, true><<<grid, 320, oz_smem_bytes(), st>>>(base, gt);
    else
      tc_gemm_kernel<KIND_I8><<<grid, 192, gemm_smem_bytes<KIND_I8>(), st>>>(base, gt);
    oz_fixup_grouped<<<pgrid, 256, 0, st>>>(fix, n);
    l = 3 + 2 * ((int)g.chunks.size() - 1);  // prep, per chunk row maxima + digits, GEMM, fixup
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    std::ostringstream s;
    s << "CUDA error in grouped tensor-core launch: " << cudaGetErrorString(e);
    return fail(QS_ECUDA, s.str());
  }
  count_launches(l);
  if (launches) *launches += l;
  return QS_OK;
}

void tc_group_release(TcGroup &g, cudaStream_t rel) {
  // Events and the aux stream go once their pending work is done (the
  // runtime defers the release); the tables after their last use on rel.
  for (cudaEvent_t e : g.ev) cudaEventDestroy(e);
  g.ev.clear();
  if (g.join) cudaEventDestroy(g.join);
  g.join = nullptr;
  if (g.aux) cudaStreamDestroy(g.aux);
  g.aux = nullptr;
  if (g.dev) cudaFreeAsync(g.dev, rel);
  g.dev = nullptr;
  g.dev_bytes = 0;
  g.image.clear();
}

}  // namespace qs
