/*
 * oracle.c — CPU restatement of QuasiStrided.jl's contraction, used ONLY as
 * test infrastructure: the checker for the device engine in tests/, the
 * engine-free reference in __graft_entry__.smoke(), and the timed CPU arm of
 * bench.py.  Nothing in the product links or calls it.
 *
 * Parity status: the reference is Julia and cannot run here (no julia
 * binary).  This restatement is pinned against the reference's own
 * known-answer tests (tests/golden/, generated by tests/golden/make_golden.py
 * from the formulas in the reference's test files), not against outputs of
 * the reference binary.
 *
 * Two entry points:
 *
 *  oracle_brute  — the engine-free definition: `_brute_ref`
 *      (test/execution/helpers.jl:6-32) and `_lo_reference`
 *      (test/helpers.jl:94-125): for every element of C, loop over every K
 *      label assignment (first K label fastest, in indA order unless an
 *      explicit K order is given), with the arithmetic of `ScalarKernel`
 *      (src/microkernels/steps.jl:27-36): acc = muladd(a, b, acc) in the
 *      compute type T, complex in the planar kernel's fused order
 *      (src/microkernels/steps.jl:121-167).  T follows `compute_type`
 *      (src/planning/plan.jl:278-285); operands are converted to T on load
 *      with conjugation = flag XOR view op (src/planning/plan.jl:176-192);
 *      the store is `axpby` with beta's Zero/One/general cases
 *      (src/microkernels/interface.jl:99-104), rounding once to eltype(C).
 *      precision = 1 evaluates the same sum in binary128 (__float128), the
 *      stand-in for the reference tests' BigFloat checks.
 *
 *  oracle_nest_f64 — a restatement of the reference's five-loop nest for a
 *      real Float64 contraction (src/execution/nest.jl:7-191): N blocks x
 *      K blocks (pack B) x M blocks (pack A) x register tiles, beta applied
 *      on the first K block only (nest.jl:83), packed panels, an MR x NR
 *      FMA microkernel.  Parallel over M x N macro-tiles with OpenMP.  It is
 *      the CPU baseline bench.py times; rows [m_lo, m_hi) of M bound the
 *      sample.
 */
#include <math.h>
#include <quadmath.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Same layout as qs_view (include/qsgpu.h); host pointers here. */
typedef struct {
  void *data;
  int64_t length;
  int64_t offset;
  const int64_t *size;
  const int64_t *strides;
  int32_t ndim;
  int32_t eltype; /* 0 F32, 1 F64, 2 C32, 3 C64 */
  int32_t op;     /* 0 identity, 1 conj, 2 transpose, 3 adjoint */
  int32_t reserved;
} or_view;

enum { OR_F32 = 0, OR_F64 = 1, OR_C32 = 2, OR_C64 = 3 };

static int is_cplx(int t) { return t == OR_C32 || t == OR_C64; }
static int is_dbl(int t) { return t == OR_F64 || t == OR_C64; }
static int op_conj(int op) { return op == 1 || op == 3; }

#define MAXL 64

typedef struct {
  int nl;               /* number of distinct labels */
  int64_t lab[MAXL];    /* label values */
  int64_t ext[MAXL];    /* extents */
  int64_t sA[MAXL], sB[MAXL], sC[MAXL]; /* stride of each label per operand (0 if absent) */
  int nk;
  int kidx[MAXL];       /* K label indices (into lab), in enumeration order */
  int nc;
  int cidx[MAXL];       /* C's labels in C axis order */
} labelset;

static int find(int64_t l, const int64_t *ind, int n) {
  for (int i = 0; i < n; ++i)
    if (ind[i] == l) return i;
  return -1;
}

static int build_labels(labelset *L, const or_view *A, const int64_t *indA, const or_view *B,
                        const int64_t *indB, const or_view *C, const int64_t *indC,
                        const int64_t *korder, int nkorder) {
  memset(L, 0, sizeof(*L));
  const or_view *vs[3] = {A, B, C};
  const int64_t *is[3] = {indA, indB, indC};
  for (int o = 0; o < 3; ++o) {
    for (int d = 0; d < vs[o]->ndim; ++d) {
      int64_t l = is[o][d];
      int k = -1;
      for (int i = 0; i < L->nl; ++i)
        if (L->lab[i] == l) k = i;
      if (k < 0) {
        if (L->nl >= MAXL) return -1;
        k = L->nl++;
        L->lab[k] = l;
        L->ext[k] = vs[o]->size[d];
      } else if (L->ext[k] != vs[o]->size[d]) {
        return -2;
      }
      int64_t s = vs[o]->strides[d];
      if (o == 0) L->sA[k] = s;
      if (o == 1) L->sB[k] = s;
      if (o == 2) L->sC[k] = s;
    }
  }
  /* K labels: in A and B but not C; indA order unless korder is given. */
  if (korder && nkorder > 0) {
    for (int i = 0; i < nkorder; ++i) {
      for (int k = 0; k < L->nl; ++k)
        if (L->lab[k] == korder[i]) L->kidx[L->nk++] = k;
    }
  } else {
    for (int d = 0; d < A->ndim; ++d) {
      int64_t l = indA[d];
      if (find(l, indB, B->ndim) >= 0 && find(l, indC, C->ndim) < 0) {
        for (int k = 0; k < L->nl; ++k)
          if (L->lab[k] == l) L->kidx[L->nk++] = k;
      }
    }
  }
  for (int d = 0; d < C->ndim; ++d)
    for (int k = 0; k < L->nl; ++k)
      if (L->lab[k] == indC[d]) L->cidx[L->nc++] = k;
  return 0;
}

/* ------------------------------------------------------------- loads ---- */

static double ld_re(const or_view *v, int64_t i) {
  switch (v->eltype) {
    case OR_F32: return ((const float *)v->data)[i];
    case OR_F64: return ((const double *)v->data)[i];
    case OR_C32: return ((const float *)v->data)[2 * i];
    default: return ((const double *)v->data)[2 * i];
  }
}
static double ld_im(const or_view *v, int64_t i) {
  switch (v->eltype) {
    case OR_C32: return ((const float *)v->data)[2 * i + 1];
    case OR_C64: return ((const double *)v->data)[2 * i + 1];
    default: return 0.0;
  }
}

/* --------------------------------------------------- generic arithmetic --- */
/* One instantiation per real type R of the compute type.  `CVT(x)` rounds a
 * stored value (exactly representable as double) to R, as convert(T, x). */

#define DEFINE_BRUTE(NAME, R, FMA, CVT)                                                       \
  static void NAME(const labelset *L, const or_view *C, const or_view *A, const or_view *B,   \
                   int cplx, int cA, int cB, const double *alpha, const double *beta,         \
                   int beta_case, int64_t c_lo, int64_t c_hi, int TCdbl) {                    \
    R ar_ = CVT(alpha[0]), ai_ = CVT(alpha[1]), br_ = CVT(beta[0]), bi_ = CVT(beta[1]);      \
    int64_t nC = 1;                                                                           \
    for (int d = 0; d < C->ndim; ++d) nC *= C->size[d];                                      \
    if (c_hi > nC) c_hi = nC;                                                                 \
    for (int64_t c = c_lo; c < c_hi; ++c) {                                                   \
      int64_t r = c, oA = A->offset, oB = B->offset, oC = C->offset;                          \
      for (int d = 0; d < L->nc; ++d) {                                                       \
        int k = L->cidx[d];                                                                   \
        int64_t x = r % L->ext[k];                                                            \
        r /= L->ext[k];                                                                       \
        oA += x * L->sA[k];                                                                   \
        oB += x * L->sB[k];                                                                   \
        oC += x * L->sC[k];                                                                   \
      }                                                                                       \
      R accr = 0, acci = 0;                                                                   \
      int64_t nK = 1;                                                                         \
      for (int d = 0; d < L->nk; ++d) nK *= L->ext[L->kidx[d]];                               \
      int64_t xk[MAXL];                                                                       \
      memset(xk, 0, sizeof(xk));                                                              \
      int64_t kA = 0, kB = 0;                                                                 \
      for (int64_t q = 0; q < nK; ++q) {                                                      \
        R a_r = CVT(ld_re(A, oA + kA)), b_r = CVT(ld_re(B, oB + kB));                         \
        if (!cplx) {                                                                          \
          accr = FMA(a_r, b_r, accr);                                                         \
        } else {                                                                              \
          R a_i = CVT(ld_im(A, oA + kA)), b_i = CVT(ld_im(B, oB + kB));                       \
          if (cA) a_i = -a_i;                                                                 \
          if (cB) b_i = -b_i;                                                                 \
          R nr = FMA(-a_i, b_i, FMA(a_r, b_r, accr));                                         \
          R ni = FMA(a_i, b_r, FMA(a_r, b_i, acci));                                          \
          accr = nr;                                                                          \
          acci = ni;                                                                          \
        }                                                                                     \
        for (int d = 0; d < L->nk; ++d) {                                                     \
          int k = L->kidx[d];                                                                 \
          if (xk[d] < L->ext[k] - 1) {                                                        \
            ++xk[d];                                                                          \
            kA += L->sA[k];                                                                   \
            kB += L->sB[k];                                                                   \
            break;                                                                            \
          }                                                                                   \
          kA -= (L->ext[k] - 1) * L->sA[k];                                                   \
          kB -= (L->ext[k] - 1) * L->sB[k];                                                   \
          xk[d] = 0;                                                                          \
        }                                                                                     \
      }                                                                                       \
      R outr, outi = 0;                                                                       \
      if (!cplx) {                                                                            \
        if (beta_case == 0) outr = ar_ * accr;                                                \
        else {                                                                                \
          R old = CVT(ld_re(C, oC));                                                          \
          outr = beta_case == 1 ? FMA(ar_, accr, old) : FMA(ar_, accr, br_ * old);            \
        }                                                                                     \
      } else {                                                                                \
        R pr = ar_ * accr - ai_ * acci, pi = ar_ * acci + ai_ * accr;                         \
        if (beta_case == 0) {                                                                 \
          outr = pr;                                                                          \
          outi = pi;                                                                          \
        } else {                                                                              \
          R olr = CVT(ld_re(C, oC)), oli = CVT(ld_im(C, oC));                                 \
          if (beta_case == 1) {                                                               \
            outr = pr + olr;                                                                  \
            outi = pi + oli;                                                                  \
          } else {                                                                            \
            outr = pr + (br_ * olr - bi_ * oli);                                              \
            outi = pi + (br_ * oli + bi_ * olr);                                              \
          }                                                                                   \
        }                                                                                     \
      }                                                                                       \
      switch (C->eltype) {                                                                    \
        case OR_F32: ((float *)C->data)[oC] = (float)outr; break;                             \
        case OR_F64: ((double *)C->data)[oC] = (double)outr; break;                           \
        case OR_C32:                                                                          \
          ((float *)C->data)[2 * oC] = (float)outr;                                           \
          ((float *)C->data)[2 * oC + 1] = (float)outi;                                        \
          break;                                                                              \
        default:                                                                              \
          ((double *)C->data)[2 * oC] = (double)outr;                                         \
          ((double *)C->data)[2 * oC + 1] = (double)outi;                                     \
      }                                                                                       \
      (void)TCdbl;                                                                            \
    }                                                                                         \
  }

#define CVT_F(x) ((float)(x))
#define CVT_D(x) ((double)(x))
#define CVT_Q(x) ((__float128)(x))
DEFINE_BRUTE(brute_f32, float, fmaf, CVT_F)
DEFINE_BRUTE(brute_f64, double, fma, CVT_D)
DEFINE_BRUTE(brute_f128, __float128, fmaq, CVT_Q)

static int beta_case_of(const double *beta, int dbl) {
  double re = beta[0], im = beta[1];
  if (!dbl) {
    re = (double)(float)re;
    im = (double)(float)im;
  }
  if (re == 0.0 && im == 0.0) return 0;
  if (re == 1.0 && im == 0.0) return 1;
  return 2;
}

/* Returns 0 on success, <0 on malformed input.  accumulator: 0 none,
 * 1 Float32, 2 Float64.  precision: 0 the compute type, 1 binary128.
 * Elements [c_lo, c_hi) of C (linear order of C's axes) are computed. */
int oracle_brute(const or_view *C, const double *alpha, const or_view *A, const int64_t *indA,
                 const or_view *B, const int64_t *indB, const double *beta,
                 const int64_t *indC, int conjA, int conjB, int accumulator,
                 const int64_t *korder, int nkorder, int precision, int64_t c_lo,
                 int64_t c_hi, int nthreads) {
  labelset L;
  int rc = build_labels(&L, A, indA, B, indB, C, indC, korder, nkorder);
  if (rc) return rc;
  int cplx = is_cplx(A->eltype) || is_cplx(B->eltype) || is_cplx(C->eltype);
  int dbl = is_dbl(A->eltype) || is_dbl(B->eltype) || is_dbl(C->eltype);
  if (accumulator == 1) dbl = 0;
  if (accumulator == 2) dbl = 1;
  int cA = is_cplx(A->eltype) && ((conjA != 0) != op_conj(A->op));
  int cB = is_cplx(B->eltype) && ((conjB != 0) != op_conj(B->op));
  double al[2] = {alpha[0], cplx ? alpha[1] : 0.0};
  double be[2] = {beta[0], cplx ? beta[1] : 0.0};
  int bc = beta_case_of(be, dbl || precision == 1);
  int64_t nC = 1;
  for (int d = 0; d < C->ndim; ++d) nC *= C->size[d];
  if (c_hi < 0 || c_hi > nC) c_hi = nC;
  if (c_lo < 0) c_lo = 0;
  if (nthreads < 1) nthreads = 1;
  int64_t total = c_hi - c_lo;
  int64_t chunk = (total + nthreads - 1) / (nthreads > 0 ? nthreads : 1);
  if (chunk < 1) chunk = 1;
#pragma omp parallel for num_threads(nthreads) schedule(static)
  for (int64_t t = 0; t < nthreads; ++t) {
    int64_t lo = c_lo + t * chunk, hi = lo + chunk;
    if (hi > c_hi) hi = c_hi;
    if (lo >= hi) continue;
    if (precision == 1)
      brute_f128(&L, C, A, B, cplx, cA, cB, al, be, bc, lo, hi, 1);
    else if (dbl)
      brute_f64(&L, C, A, B, cplx, cA, cB, al, be, bc, lo, hi, 1);
    else
      brute_f32(&L, C, A, B, cplx, cA, cB, al, be, bc, lo, hi, 0);
  }
  return 0;
}

/* ------------------------------------------------------------ the nest --- */
/* Real Float64 restatement of nest!/pack_block!/SIMDKernel for the CPU
 * baseline.  M labels = in A and C, N labels = in B and C, both in C-stride
 * order (order_free_labels), K labels in indA order.  Blocking constants of
 * the reference's fallback blocking for an 8x6 Float64 tile. */

#define NR_MR 8
#define NR_NR 6

static void fill_offsets(int D, const int64_t *len, const int64_t *st, int64_t first,
                         int64_t count, int64_t *out) {
  int64_t x[MAXL];
  int64_t r = first, off = 0;
  for (int d = 0; d < D; ++d) {
    x[d] = r % len[d];
    r /= len[d];
    off += x[d] * st[d];
  }
  for (int64_t t = 0; t < count; ++t) {
    out[t] = off;
    for (int d = 0; d < D; ++d) {
      if (x[d] < len[d] - 1) {
        ++x[d];
        off += st[d];
        break;
      }
      off -= (len[d] - 1) * st[d];
      x[d] = 0;
    }
  }
}

static int cmp_abs_stride_key;
typedef struct {
  int64_t key;
  int pos;
  int lab;
} skey;
static int cmp_skey(const void *a, const void *b) {
  const skey *x = a, *y = b;
  if (x->key != y->key) return x->key < y->key ? -1 : 1;
  return x->pos - y->pos; /* stable */
}

int oracle_nest_f64(const or_view *C, double alpha, const or_view *A, const int64_t *indA,
                    const or_view *B, const int64_t *indB, double beta, const int64_t *indC,
                    int64_t m_lo, int64_t m_hi, int nthreads) {
  (void)cmp_abs_stride_key;
  if (A->eltype != OR_F64 || B->eltype != OR_F64 || C->eltype != OR_F64) return -3;
  labelset L;
  int rc = build_labels(&L, A, indA, B, indB, C, indC, NULL, 0);
  if (rc) return rc;
  /* M and N labels ordered by |C stride| (stable). */
  skey mk[MAXL], nk[MAXL];
  int nm = 0, nn = 0;
  for (int d = 0; d < C->ndim; ++d) {
    int64_t l = indC[d];
    int k = -1;
    for (int i = 0; i < L.nl; ++i)
      if (L.lab[i] == l) k = i;
    int64_t s = C->strides[d] < 0 ? -C->strides[d] : C->strides[d];
    if (find(l, indA, A->ndim) >= 0) mk[nm++] = (skey){s, d, k};
    else nk[nn++] = (skey){s, d, k};
  }
  qsort(mk, nm, sizeof(skey), cmp_skey);
  qsort(nk, nn, sizeof(skey), cmp_skey);
  int64_t mlen[MAXL], mA[MAXL], mC[MAXL], nlen[MAXL], nB[MAXL], nC[MAXL], klen[MAXL], kA[MAXL],
      kB[MAXL];
  int64_t M = 1, N = 1, K = 1;
  for (int i = 0; i < nm; ++i) {
    mlen[i] = L.ext[mk[i].lab];
    mA[i] = L.sA[mk[i].lab];
    mC[i] = L.sC[mk[i].lab];
    M *= mlen[i];
  }
  for (int i = 0; i < nn; ++i) {
    nlen[i] = L.ext[nk[i].lab];
    nB[i] = L.sB[nk[i].lab];
    nC[i] = L.sC[nk[i].lab];
    N *= nlen[i];
  }
  for (int i = 0; i < L.nk; ++i) {
    klen[i] = L.ext[L.kidx[i]];
    kA[i] = L.sA[L.kidx[i]];
    kB[i] = L.sB[L.kidx[i]];
    K *= klen[i];
  }
  if (m_hi < 0 || m_hi > M) m_hi = M;
  if (m_lo < 0) m_lo = 0;
  if (M == 0 || N == 0 || m_lo >= m_hi) return 0;
  int64_t *offMA = malloc(sizeof(int64_t) * M), *offMC = malloc(sizeof(int64_t) * M);
  int64_t *offNB = malloc(sizeof(int64_t) * N), *offNC = malloc(sizeof(int64_t) * N);
  int64_t *offKA = malloc(sizeof(int64_t) * (K ? K : 1)), *offKB = malloc(sizeof(int64_t) * (K ? K : 1));
  fill_offsets(nm, mlen, mA, 0, M, offMA);
  fill_offsets(nm, mlen, mC, 0, M, offMC);
  fill_offsets(nn, nlen, nB, 0, N, offNB);
  fill_offsets(nn, nlen, nC, 0, N, offNC);
  if (K) {
    fill_offsets(L.nk, klen, kA, 0, K, offKA);
    fill_offsets(L.nk, klen, kB, 0, K, offKB);
  }
  const double *Ad = (const double *)A->data + A->offset;
  const double *Bd = (const double *)B->data + B->offset;
  double *Cd = (double *)C->data + C->offset;
  const int64_t MC = 96, KC = 256, NC = 576; /* fallback-like blocking */
  int64_t mblocks = (m_hi - m_lo + MC - 1) / MC, nblocks = (N + NC - 1) / NC;
  if (nthreads < 1) nthreads = 1;
#pragma omp parallel num_threads(nthreads)
  {
    double *pa = aligned_alloc(64, sizeof(double) * MC * KC);
    double *pb = aligned_alloc(64, sizeof(double) * KC * (NC + NR_NR));
#pragma omp for collapse(2) schedule(dynamic)
    for (int64_t nb = 0; nb < nblocks; ++nb) {
      for (int64_t mb = 0; mb < mblocks; ++mb) {
        int64_t n0 = nb * NC, nlen_b = N - n0 < NC ? N - n0 : NC;
        int64_t m0 = m_lo + mb * MC, mlen_b = m_hi - m0 < MC ? m_hi - m0 : MC;
        int first = 1;
        for (int64_t k0 = 0; k0 < K || (K == 0 && first); k0 += KC) {
          int64_t klen_b = K - k0 < KC ? K - k0 : KC;
          if (K == 0) klen_b = 0;
          double bet = first ? beta : 1.0;
          /* pack B: slivers of NR columns, K-major within a sliver */
          int64_t ntl = (nlen_b + NR_NR - 1) / NR_NR;
          for (int64_t t = 0; t < ntl; ++t)
            for (int64_t p = 0; p < klen_b; ++p)
              for (int j = 0; j < NR_NR; ++j) {
                int64_t n = n0 + t * NR_NR + j;
                pb[(t * klen_b + p) * NR_NR + j] = n < n0 + nlen_b ? Bd[offNB[n] + offKB[k0 + p]] : 0.0;
              }
          int64_t mtl = (mlen_b + NR_MR - 1) / NR_MR;
          for (int64_t t = 0; t < mtl; ++t)
            for (int64_t p = 0; p < klen_b; ++p)
              for (int i = 0; i < NR_MR; ++i) {
                int64_t m = m0 + t * NR_MR + i;
                pa[(t * klen_b + p) * NR_MR + i] = m < m0 + mlen_b ? Ad[offMA[m] + offKA[k0 + p]] : 0.0;
              }
          for (int64_t tn = 0; tn < ntl; ++tn)
            for (int64_t tm = 0; tm < mtl; ++tm) {
              double acc[NR_NR][NR_MR];
              memset(acc, 0, sizeof(acc));
              const double *a = pa + tm * klen_b * NR_MR, *b = pb + tn * klen_b * NR_NR;
              for (int64_t p = 0; p < klen_b; ++p)
                for (int j = 0; j < NR_NR; ++j)
                  for (int i = 0; i < NR_MR; ++i)
                    acc[j][i] = fma(a[p * NR_MR + i], b[p * NR_NR + j], acc[j][i]);
              for (int j = 0; j < NR_NR; ++j) {
                int64_t n = n0 + tn * NR_NR + j;
                if (n >= n0 + nlen_b) break;
                for (int i = 0; i < NR_MR; ++i) {
                  int64_t m = m0 + tm * NR_MR + i;
                  if (m >= m0 + mlen_b) break;
                  double *c = Cd + offMC[m] + offNC[n];
                  if (bet == 0.0) *c = alpha * acc[j][i];
                  else if (bet == 1.0) *c = fma(alpha, acc[j][i], *c);
                  else *c = fma(alpha, acc[j][i], bet * *c);
                }
              }
            }
          first = 0;
          if (K == 0) break;
        }
      }
    }
    free(pa);
    free(pb);
  }
  free(offMA); free(offMC); free(offNB); free(offNC); free(offKA); free(offKB);
  return 0;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
