// Device-side scalar helpers shared by the kernels: the compute types, loads
// that convert a stored element to the compute type with conjugation on load
// (the packing transform of src/packing/pack.jl:43-59), and the alpha/beta
// store with its Zero/One/beta cases (src/microkernels/interface.jl:99-104),
// rounding once to eltype(C).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/qsgpu.h"

namespace qs {

template <class R>
struct cplx {
  R re, im;
};

template <class T> struct real_of { using type = T; };
template <class R> struct real_of<cplx<R>> { using type = R; };
template <class T> struct is_cplx { static constexpr bool value = false; };
template <class R> struct is_cplx<cplx<R>> { static constexpr bool value = true; };

// Device launch parameters of a contraction: operand bases, eltypes and the
// offset tables of the M/N/K groups (maps as in qs::Group).
struct Operands {
  const void *A;
  const void *B;
  void *C;
  int64_t Abase, Bbase, Cbase;
  int TA, TB, TC;
  int conjA, conjB;
  const int64_t *offMA, *offMC, *offNB, *offNC, *offKA, *offKB;
  int64_t M, N, K;
  // Batch labels: entry b adds offBatch[b], [P + b], [2P + b] to the A, B and
  // C bases (nullptr and P = 1 without batch labels).
  const int64_t *offBatch = nullptr;
  int64_t P = 1;
};

// The operands of batch entry b.
__device__ __forceinline__ Operands batch_entry(const Operands &op, int64_t b) {
  Operands o = op;
  if (op.offBatch) {
    o.Abase += op.offBatch[b];
    o.Bbase += op.offBatch[op.P + b];
    o.Cbase += op.offBatch[2 * op.P + b];
  }
  return o;
}

// Stored element (any supported eltype) -> real compute type.
template <class R>
__device__ __forceinline__ R load_real(const void *base, int64_t idx, int et) {
  if (et == QS_F64) return (R)__ldg((const double *)base + idx);
  return (R)__ldg((const float *)base + idx);
}

template <class T>
struct Loader;

template <>
struct Loader<float> {
  static __device__ __forceinline__ float load(const void *b, int64_t i, int et, int) {
    return load_real<float>(b, i, et);
  }
};
template <>
struct Loader<double> {
  static __device__ __forceinline__ double load(const void *b, int64_t i, int et, int) {
    return load_real<double>(b, i, et);
  }
};
template <class R>
struct Loader<cplx<R>> {
  static __device__ __forceinline__ cplx<R> load(const void *b, int64_t i, int et, int conj) {
    cplx<R> v;
    switch (et) {
      case QS_F32: v.re = (R)__ldg((const float *)b + i); v.im = 0; return v;
      case QS_F64: v.re = (R)__ldg((const double *)b + i); v.im = 0; return v;
      case QS_C32: {
        float2 x = __ldg((const float2 *)b + i);
        v.re = (R)x.x;
        v.im = (R)(conj ? -x.y : x.y);
        return v;
      }
      default: {
        const double *p = (const double *)b + 2 * i;
        v.re = (R)__ldg(p);
        double im = __ldg(p + 1);
        v.im = (R)(conj ? -im : im);
        return v;
      }
    }
  }
};

// C's stored element -> compute type (never conjugated).
template <class T>
__device__ __forceinline__ T load_c(const void *b, int64_t i, int et) {
  if constexpr (is_cplx<T>::value) {
    using R = typename real_of<T>::type;
    T v;
    if (et == QS_C32) {
      float2 x = ((const float2 *)b)[i];
      v.re = (R)x.x;
      v.im = (R)x.y;
    } else {
      const double *p = (const double *)b + 2 * i;
      v.re = (R)p[0];
      v.im = (R)p[1];
    }
    return v;
  } else {
    if (et == QS_F64) return (T)((const double *)b)[i];
    return (T)((const float *)b)[i];
  }
}

template <class T>
__device__ __forceinline__ void store_c(void *b, int64_t i, int et, T v) {
  if constexpr (is_cplx<T>::value) {
    if (et == QS_C32) {
      ((float2 *)b)[i] = make_float2((float)v.re, (float)v.im);
    } else {
      double *p = (double *)b + 2 * i;
      p[0] = (double)v.re;
      p[1] = (double)v.im;
    }
  } else {
    if (et == QS_F64) ((double *)b)[i] = (double)v;
    else ((float *)b)[i] = (float)v;
  }
}

// Arithmetic in the compute type.
template <class R>
__device__ __forceinline__ R cmul(R a, R b) { return a * b; }
template <class R>
__device__ __forceinline__ cplx<R> cmul(cplx<R> a, cplx<R> b) {
  cplx<R> r;
  r.re = a.re * b.re - a.im * b.im;
  r.im = a.re * b.im + a.im * b.re;
  return r;
}
template <class R>
__device__ __forceinline__ R cfma(R a, R b, R c) { return fma(a, b, c); }
// Complex multiply-add in the planar kernel's fused order
// (src/microkernels/steps.jl:121-167):
//   re = muladd(-ai, bi, muladd(ar, br, c.re))
//   im = muladd( ai, br, muladd(ar, bi, c.im))
template <class R>
__device__ __forceinline__ cplx<R> cfma(cplx<R> a, cplx<R> b, cplx<R> c) {
  cplx<R> r;
  r.re = fma(-a.im, b.im, fma(a.re, b.re, c.re));
  r.im = fma(a.im, b.re, fma(a.re, b.im, c.im));
  return r;
}
template <class R>
__device__ __forceinline__ R czero() { return (R)0; }
template <class T>
__device__ __forceinline__ T tzero() {
  if constexpr (is_cplx<T>::value) {
    T z;
    z.re = 0;
    z.im = 0;
    return z;
  } else {
    return (T)0;
  }
}

// Scalars for a launch: alpha/beta in the compute type plus beta's case
// (0: Zero, 1: One, 2: general), src/microkernels/interface.jl:99.
template <class T>
struct Scalars {
  T alpha, beta;
  int beta_case;
};

// axpby (src/microkernels/interface.jl:102-104): Zero ignores old; One is
// muladd(alpha, r, old); general is muladd(alpha, r, beta*old).
template <class T>
__device__ __forceinline__ T axpby(const Scalars<T> &s, T r, T old) {
  if (s.beta_case == 0) return cmul(s.alpha, r);
  if (s.beta_case == 1) return cfma(s.alpha, r, old);
  return cfma(s.alpha, r, cmul(s.beta, old));
}

// Host: alpha/beta ({re, im} doubles) in compute type T.
template <class T>
inline Scalars<T> make_scalars(const double *alpha, const double *beta, int beta_case) {
  Scalars<T> s;
  if constexpr (is_cplx<T>::value) {
    using R = typename real_of<T>::type;
    s.alpha.re = (R)alpha[0];
    s.alpha.im = (R)alpha[1];
    s.beta.re = (R)beta[0];
    s.beta.im = (R)beta[1];
  } else {
    s.alpha = (T)alpha[0];
    s.beta = (T)beta[0];
  }
  s.beta_case = beta_case;
  return s;
}

// One problem of a grouped gather-GEMM launch: a CTA finds the job whose
// block range holds its index and runs tile (lb % gx, lb / gx) of it.
template <class T>
struct NativeJob {
  Operands op;
  Scalars<T> s;
  int a_mfast, b_nfast;
  int gx;  // tiles along M
  int block_start;
};

}  // namespace qs
