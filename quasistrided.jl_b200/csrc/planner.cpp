// Host-side planner: labels -> M/N/K groups -> orientation -> path -> method.
//
// Restates the planning stages of QuasiStrided.jl's `planned`
// (src/planning/plan.jl:197-262) for a device engine:
//   compute_type          src/planning/plan.jl:278-285
//   conjugation folding   src/planning/plan.jl:176-192, 210-221
//   classify_labels       src/planning/labels.jl:28-102
//   order_free_labels     src/planning/labels.jl:109-115
//   leading_unit_run      src/planning/labels.jl:249-263
//   AxisGroup             src/layout/axis_group.jl:5-73
//   order_contract_labels src/planning/labels.jl:215-243 (device cost model)
//   prefer_swap           src/planning/labels.jl:269-270 (device rule)
//   select_path           src/planning/plan.jl:395-412
// The CPU cache-blocking and register-shape menus (src/planning/blocking.jl,
// src/planning/kernel_selection.jl) have no device counterpart: the tile
// shapes are fixed by the tensor-core kernels and the autotuner.
#include <algorithm>
#include <cstring>
#include <numeric>
#include <sstream>

#include "qs_internal.h"

namespace qs {

static thread_local Status g_last;

void set_error(int code, const std::string &msg) {
  g_last.code = code;
  g_last.msg = msg;
}
int fail(int code, const std::string &msg) {
  set_error(code, msg);
  return code;
}

const char *eltype_name(int t) {
  switch (t) {
    case QS_F32: return "Float32";
    case QS_F64: return "Float64";
    case QS_C32: return "ComplexF32";
    case QS_C64: return "ComplexF64";
  }
  return "unknown";
}

// ---------------------------------------------------------------- Group ---

void Group::offset_range(int p, int64_t &lo, int64_t &hi) const {
  lo = 0;
  hi = 0;
  for (int d = 0; d < D; ++d) {
    if (len[d] == 0) {
      lo = 0;
      hi = -1;
      return;
    }
  }
  for (int d = 0; d < D; ++d) {
    int64_t span = (len[d] - 1) * st[p][d];
    if (span < 0) lo += span; else hi += span;
  }
}

int64_t Group::ramp_step(int p, bool &ok) const {
  ok = true;
  int64_t step = 0, run = 1;
  bool started = false;
  for (int d = 0; d < D; ++d) {
    int64_t L = len[d];
    if (L == 0) return 0;
    if (L == 1) continue;
    int64_t S = st[p][d];
    if (!started) {
      step = S;
      run = L;
      started = true;
    } else {
      __int128 want = (__int128)run * (__int128)step;
      if (want != (__int128)S) {
        ok = false;
        return 0;
      }
      run *= L;
    }
  }
  return step;
}

void Group::fill_offsets(int p, int64_t first, int64_t count, int64_t *out) const {
  if (count <= 0) return;
  int64_t x[kMaxRank];
  int64_t r = first, off = 0;
  for (int d = 0; d < D; ++d) {
    int64_t L = len[d];
    x[d] = r % L;
    r /= L;
    off += x[d] * st[p][d];
  }
  for (int64_t t = 0;;) {
    out[t++] = off;
    if (t == count) break;
    for (int d = 0; d < D; ++d) {
      if (x[d] < len[d] - 1) {
        ++x[d];
        off += st[p][d];
        break;
      }
      off -= (len[d] - 1) * st[p][d];
      x[d] = 0;
    }
  }
}

// ------------------------------------------------------------- helpers ---

static bool checked_mul(int64_t a, int64_t b, int64_t &out) {
  return !__builtin_mul_overflow(a, b, &out);
}
static bool checked_add(int64_t a, int64_t b, int64_t &out) {
  return !__builtin_add_overflow(a, b, &out);
}

static int find_label(int64_t lbl, const int64_t *ind, int n) {
  for (int i = 0; i < n; ++i)
    if (ind[i] == lbl) return i;
  return -1;
}

static std::string tuple_str(const int64_t *ind, int n) {
  std::ostringstream s;
  s << "(";
  for (int i = 0; i < n; ++i) s << (i ? ", " : "") << ind[i];
  if (n == 1) s << ",";
  s << ")";
  return s.str();
}

static bool all_unique(const int64_t *ind, int n) {
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j)
      if (ind[i] == ind[j]) return false;
  return true;
}

// validate_axis_group_bounds (src/layout/axis_group.jl:27-41): the
// cardinality and every map's offset range fit in Int64.
static int validate_group(const Group &g) {
  for (int d = 0; d < g.D; ++d)
    if (g.len[d] == 0) return QS_OK;
  int64_t q = 1;
  for (int d = 0; d < g.D; ++d)
    if (!checked_mul(q, g.len[d], q))
      return fail(QS_EINVAL, "OverflowError: axis group cardinality overflows Int64");
  for (int p = 0; p < 2; ++p) {
    int64_t acc = 0;
    for (int d = 0; d < g.D; ++d) {
      if (g.len[d] <= 1) continue;
      int64_t s = g.st[p][d];
      if (s == INT64_MIN) return fail(QS_EINVAL, "OverflowError: stride overflows Int64");
      int64_t t;
      if (!checked_mul(g.len[d] - 1, s < 0 ? -s : s, t) || !checked_add(acc, t, acc))
        return fail(QS_EINVAL, "OverflowError: axis group offset range overflows Int64");
    }
  }
  return QS_OK;
}

// AxisGroup(labels, (ind1, v1), (ind2, v2)) (src/layout/axis_group.jl:50-69).
static int make_group(Group &g, const int64_t *labels, int D, const int64_t *ind1,
                      const qs_view *v1, const int64_t *ind2, const qs_view *v2) {
  g.D = D;
  for (int d = 0; d < D; ++d) {
    int p1 = find_label(labels[d], ind1, v1->ndim);
    int p2 = find_label(labels[d], ind2, v2->ndim);
    int64_t l1 = v1->size[p1], l2 = v2->size[p2];
    if (l1 != l2) {
      std::ostringstream s;
      s << "DimensionMismatch: label " << labels[d] << " has mismatched axis length: " << l1
        << " vs " << l2;
      return fail(QS_EDIM, s.str());
    }
    g.len[d] = l1;
    g.st[0][d] = v1->strides[p1];
    g.st[1][d] = v2->strides[p2];
    g.label[d] = labels[d];
  }
  return validate_group(g);
}

// Stable sort of free labels by |stride| in C (src/planning/labels.jl:109-115).
static void order_free(int64_t *labels, int D, const int64_t *indC, const qs_view *C) {
  std::vector<int> idx(D);
  std::iota(idx.begin(), idx.end(), 0);
  std::vector<int64_t> key(D), tmp(labels, labels + D);
  for (int d = 0; d < D; ++d) {
    int64_t s = C->strides[find_label(labels[d], indC, C->ndim)];
    key[d] = s < 0 ? -s : s;
  }
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return key[a] < key[b]; });
  for (int d = 0; d < D; ++d) labels[d] = tmp[idx[d]];
}

// leading_unit_run (src/planning/labels.jl:249-263).
static int64_t leading_unit_run(const int64_t *labels, int D, const int64_t *indC,
                                const qs_view *C) {
  int64_t run = 1;
  for (int d = 0; d < D; ++d) {
    int p = find_label(labels[d], indC, C->ndim);
    int64_t L = C->size[p];
    if (L == 1) continue;
    if (L == 0) return 0;
    if (C->strides[p] != run) break;
    run *= L;
  }
  return run;
}

// Device K-order cost (the counterpart of k_order_cost,
// src/planning/labels.jl:172-211).  The device gathers an operand either
// along its free composite (when that is unit-stride: every K order reads
// whole 32-byte sectors) or along K, where a fastest K axis of stride s
// spends one sector per element once s*size exceeds a sector.
static double k_cost(const std::vector<int> &perm, const int64_t *klen, const int64_t *kst,
                     bool free_unit, int64_t n, int S) {
  if (free_unit) return (double)n;
  int kfast = -1;
  for (int i : perm)
    if (klen[i] > 1) {
      kfast = i;
      break;
    }
  if (kfast < 0) return 0.0;
  int64_t s = kst[kfast] < 0 ? -kst[kfast] : kst[kfast];
  double amp = (s * S <= 32) ? 1.0 : std::min<double>(32.0 / S, (double)klen[kfast]);
  if (amp < 1.0) amp = 1.0;
  return (double)n * amp;
}

static bool free_unit_stride(const int64_t *labels, int D, const int64_t *ind, const qs_view *v) {
  for (int d = 0; d < D; ++d) {
    int p = find_label(labels[d], ind, v->ndim);
    if (v->size[p] == 1) continue;
    int64_t s = v->strides[p];
    return s == 1 || s == -1;
  }
  return false;
}

// ----------------------------------------------------------------- plan ---

int check_bounds(const qs_plan *p, bool reads_ab) {
  // bmap: which batch map adds to the range (0 = M-role operand, 1 = N-role
  // operand, 2 = C); an unbatched plan's batch range is [0, 0].
  auto span = [p](int64_t base, const Group &g1, int p1, const Group &g2, int p2, int bmap, int64_t len,
                  const char *which) -> int {
    int64_t rlo, rhi, clo, chi, blo = 0, bhi = 0;
    g1.offset_range(p1, rlo, rhi);
    g2.offset_range(p2, clo, chi);
    if (rhi < rlo || chi < clo) return QS_OK;
    if (p->batched) {
      if (bmap == 2) p->bgc.offset_range(0, blo, bhi);
      else p->bg.offset_range(bmap, blo, bhi);
      if (bhi < blo) return QS_OK;
    }
    __int128 lo = (__int128)base + rlo + clo + blo, hi = (__int128)base + rhi + chi + bhi;
    if (lo >= 0 && hi <= (__int128)len - 1) return QS_OK;
    std::ostringstream s;
    s << "BoundsError: " << which << " addresses [" << (long long)lo << ", " << (long long)hi
      << "] exceed storage bounds [0, " << len - 1 << "]";
    return fail(QS_EBOUNDS, s.str());
  };
  int rc = span(p->Cbase, p->mg, 1, p->ng, 1, 2, p->Clen, "C");
  if (rc) return rc;
  if (reads_ab) {
    rc = span(p->Abase, p->mg, 0, p->kg, 0, 0, p->Alen, p->swapped ? "B" : "A");
    if (rc) return rc;
    rc = span(p->Bbase, p->ng, 0, p->kg, 1, 1, p->Blen, p->swapped ? "A" : "B");
    if (rc) return rc;
  }
  return QS_OK;
}

int validate_view(const qs_view *v, const char *name) {
  if (!v) return fail(QS_EINVAL, std::string("ArgumentError: ") + name + " is NULL");
  if (v->ndim < 0 || v->ndim > 64)
    return fail(QS_EINVAL, std::string("ArgumentError: ") + name + " has an invalid rank");
  if (v->ndim > 0 && (!v->size || !v->strides))
    return fail(QS_EINVAL, std::string("ArgumentError: ") + name + " size/strides are NULL");
  for (int d = 0; d < v->ndim; ++d)
    if (v->size[d] < 0)
      return fail(QS_EINVAL, std::string("ArgumentError: ") + name + " has a negative size");
  if (v->length < 0)
    return fail(QS_EINVAL, std::string("ArgumentError: ") + name + " has a negative length");
  if (v->eltype < QS_F32 || v->eltype > QS_C64)
    return fail(QS_EINVAL, "ArgumentError: plan_contract: eltype of " + std::string(name) +
                               " must be one of Float32, Float64, ComplexF32, ComplexF64");
  if (v->op < QS_OP_IDENTITY || v->op > QS_OP_ADJOINT)
    return fail(QS_EINVAL,
                "ArgumentError: unsupported StridedView.op: QuasiStrided folds a view's `op` "
                "into the packing transform and recognizes only identity/conj/transpose/adjoint");
  return QS_OK;
}

static bool op_conjugates(int op) { return op == QS_OP_CONJ || op == QS_OP_ADJOINT; }

int plan_host(qs_plan *p, const qs_view *C, const qs_view *A, const int64_t *indA,
              const qs_view *B, const int64_t *indB, const int64_t *indC,
              const qs_plan_options *opts) {
  int rc;
  if ((rc = validate_view(C, "C")) || (rc = validate_view(A, "A")) ||
      (rc = validate_view(B, "B")))
    return rc;
  if ((A->ndim && !indA) || (B->ndim && !indB) || (C->ndim && !indC))
    return fail(QS_EINVAL, "ArgumentError: label tuple is NULL");
  qs_plan_options o{};
  if (opts) o = *opts;
  if (o.m_block < 0 || o.k_block < 0 || o.n_block < 0)
    return fail(QS_EINVAL, "ArgumentError: m_block/k_block/n_block must be >= 1");
  if (o.accumulator < QS_ACC_NONE || o.accumulator > QS_ACC_F64)
    return fail(QS_EINVAL, "ArgumentError: accumulator must be nothing, Float32 or Float64");
  p->opts = o;
  p->host_only = (o.flags & QS_PLAN_HOST_ONLY) ? 1 : 0;

  // compute_type (src/planning/plan.jl:278-285)
  int TA = A->eltype, TB = B->eltype, TC = C->eltype;
  if (!is_complex(TC) && (is_complex(TA) || is_complex(TB))) {
    std::ostringstream s;
    s << "ArgumentError: plan_contract: a complex operand (A: " << eltype_name(TA)
      << ", B: " << eltype_name(TB) << ") needs a complex C, got " << eltype_name(TC);
    return fail(QS_EINVAL, s.str());
  }
  bool cplx = is_complex(TA) || is_complex(TB) || is_complex(TC);
  bool dbl = is_double(TA) || is_double(TB) || is_double(TC);
  if (o.accumulator == QS_ACC_F32) dbl = false;
  if (o.accumulator == QS_ACC_F64) dbl = true;
  int T = cplx ? (dbl ? QS_C64 : QS_C32) : (dbl ? QS_F64 : QS_F32);

  // A conjugated C is rejected; C must not alias A or B (plan.jl:210-219).
  if (is_complex(TC) && op_conjugates(C->op))
    return fail(QS_EINVAL,
                "ArgumentError: plan_contract: cannot write into a conjugated view; writing a "
                "conjugated output is not supported");
  auto overlaps = [](const qs_view *x, const qs_view *y) {
    if (x->length == 0 || y->length == 0 || !x->data || !y->data) return false;
    uintptr_t x0 = (uintptr_t)x->data, x1 = x0 + (uintptr_t)x->length * elsize(x->eltype);
    uintptr_t y0 = (uintptr_t)y->data, y1 = y0 + (uintptr_t)y->length * elsize(y->eltype);
    return x0 < y1 && y0 < x1;
  };
  if (overlaps(C, A) || overlaps(C, B))
    return fail(QS_EINVAL, "ArgumentError: plan_contract: C must not share memory with A or B");
  int conjA = is_complex(TA) && ((o.conjA != 0) != op_conjugates(A->op));
  int conjB = is_complex(TB) && ((o.conjB != 0) != op_conjugates(B->op));

  // classify_labels (src/planning/labels.jl:28-102)
  int NA = A->ndim, NB = B->ndim, NC = C->ndim;
  if (!all_unique(indA, NA))
    return fail(QS_EINVAL, "ArgumentError: indA has a repeated label (diagonal), not supported: " +
                               tuple_str(indA, NA));
  if (!all_unique(indB, NB))
    return fail(QS_EINVAL, "ArgumentError: indB has a repeated label (diagonal), not supported: " +
                               tuple_str(indB, NB));
  if (!all_unique(indC, NC))
    return fail(QS_EINVAL, "ArgumentError: indC has a repeated label (diagonal), not supported: " +
                               tuple_str(indC, NC));
  std::vector<int64_t> ml, nl, kl, bl;
  const bool batch_ok = (o.flags & QS_PLAN_BATCH_LABELS) != 0;
  for (int i = 0; i < NA; ++i) {
    int64_t l = indA[i];
    bool inB = find_label(l, indB, NB) >= 0, inC = find_label(l, indC, NC) >= 0;
    if (inB && inC && batch_ok) {
      bl.push_back(l);
    } else if (inB && inC) {
      std::ostringstream s;
      s << "ArgumentError: label " << l
        << " appears in indA, indB, and indC: labels present in all three operands "
           "(batch-like) are not supported";
      return fail(QS_EINVAL, s.str());
    } else if (inB) {
      kl.push_back(l);
    } else if (inC) {
      ml.push_back(l);
    } else {
      std::ostringstream s;
      s << "ArgumentError: label " << l
        << " appears only in indA (not in indB or indC): not a valid free (M) or contracted "
           "(K) label";
      return fail(QS_EINVAL, s.str());
    }
  }
  for (int i = 0; i < NB; ++i) {
    int64_t l = indB[i];
    if (find_label(l, indA, NA) >= 0) continue;
    if (find_label(l, indC, NC) >= 0) {
      nl.push_back(l);
    } else {
      std::ostringstream s;
      s << "ArgumentError: label " << l
        << " appears only in indB (not in indA or indC): not a valid free (N) or contracted "
           "(K) label";
      return fail(QS_EINVAL, s.str());
    }
  }
  for (int i = 0; i < NC; ++i) {
    int64_t l = indC[i];
    if (find_label(l, indA, NA) < 0 && find_label(l, indB, NB) < 0) {
      std::ostringstream s;
      s << "ArgumentError: label " << l << " appears in indC but not in indA or indB";
      return fail(QS_EINVAL, s.str());
    }
  }
  if ((int)ml.size() > kMaxRank || (int)nl.size() > kMaxRank || (int)kl.size() > kMaxRank ||
      (int)bl.size() > kMaxRank)
    return fail(QS_EINVAL, "ArgumentError: more than 16 labels in one composite");

  // Free label order by |C stride| and C's unit-stride runs.
  order_free(ml.data(), (int)ml.size(), indC, C);
  order_free(nl.data(), (int)nl.size(), indC, C);
  int64_t run_m = leading_unit_run(ml.data(), (int)ml.size(), indC, C);
  int64_t run_n = leading_unit_run(nl.data(), (int)nl.size(), indC, C);

  Group mg, ng, kg;
  if ((rc = make_group(mg, ml.data(), (int)ml.size(), indA, A, indC, C))) return rc;
  if ((rc = make_group(ng, nl.data(), (int)nl.size(), indB, B, indC, C))) return rc;
  // Validate K lengths in indA order first (DimensionMismatch before ordering).
  if ((rc = make_group(kg, kl.data(), (int)kl.size(), indA, A, indB, B))) return rc;
  Group bg, bgc;
  if ((rc = make_group(bg, bl.data(), (int)bl.size(), indA, A, indB, B))) return rc;
  if ((rc = make_group(bgc, bl.data(), (int)bl.size(), indC, C, indA, A))) return rc;

  // K order: indA order, sorted by A's strides, sorted by B's strides;
  // ties keep indA order (src/planning/labels.jl:215-243).
  int DK = (int)kl.size();
  if (DK > 1) {
    std::vector<int> id(DK), pa(DK), pb(DK);
    std::iota(id.begin(), id.end(), 0);
    pa = id;
    pb = id;
    int64_t absA[kMaxRank], absB[kMaxRank];
    for (int d = 0; d < DK; ++d) {
      absA[d] = kg.st[0][d] < 0 ? -kg.st[0][d] : kg.st[0][d];
      absB[d] = kg.st[1][d] < 0 ? -kg.st[1][d] : kg.st[1][d];
    }
    std::stable_sort(pa.begin(), pa.end(), [&](int a, int b) { return absA[a] < absA[b]; });
    std::stable_sort(pb.begin(), pb.end(), [&](int a, int b) { return absB[a] < absB[b]; });
    bool fa = free_unit_stride(ml.data(), (int)ml.size(), indA, A);
    bool fb = free_unit_stride(nl.data(), (int)nl.size(), indB, B);
    int64_t nA = 1, nB = 1;
    for (int d = 0; d < A->ndim; ++d) nA *= A->size[d];
    for (int d = 0; d < B->ndim; ++d) nB *= B->size[d];
    auto cost = [&](const std::vector<int> &perm) {
      return k_cost(perm, kg.len, kg.st[0], fa, nA, elsize(TA)) +
             k_cost(perm, kg.len, kg.st[1], fb, nB, elsize(TB));
    };
    std::vector<int> best = id;
    double bestc = cost(id);
    for (auto *cand : {&pa, &pb}) {
      if (*cand == best) continue;
      double c = cost(*cand);
      if (c < bestc) {
        best = *cand;
        bestc = c;
      }
    }
    if (best != id) {
      Group k2 = kg;
      for (int d = 0; d < DK; ++d) {
        k2.len[d] = kg.len[best[d]];
        k2.st[0][d] = kg.st[0][best[d]];
        k2.st[1][d] = kg.st[1][best[d]];
        k2.label[d] = kg.label[best[d]];
      }
      kg = k2;
    }
  }

  // Orientation.  The device epilogue stores a column of C per warp-lane
  // group along M, so the role with the longer unit-stride run in C takes M
  // (the device analogue of prefer_swap, src/planning/labels.jl:269-270).
  // The sum is unchanged; complex products commute exactly, so the rule
  // applies to every eltype.
  bool swap = run_m < 32 && run_n > run_m;
  p->T = T;
  p->TC = TC;
  p->Cdata = C->data;
  p->Clen = C->length;
  p->Cbase = C->offset;
  if (!swap) {
    p->TA = TA; p->TB = TB;
    p->Adata = A->data; p->Alen = A->length; p->Abase = A->offset;
    p->Bdata = B->data; p->Blen = B->length; p->Bbase = B->offset;
    p->conjA = conjA; p->conjB = conjB;
    p->mg = mg; p->ng = ng; p->kg = kg;
  } else {
    p->TA = TB; p->TB = TA;
    p->Adata = B->data; p->Alen = B->length; p->Abase = B->offset;
    p->Bdata = A->data; p->Blen = A->length; p->Bbase = A->offset;
    p->conjA = conjB; p->conjB = conjA;
    p->mg = ng; p->ng = mg;
    Group k2 = kg;
    for (int d = 0; d < kg.D; ++d) {
      k2.st[0][d] = kg.st[1][d];
      k2.st[1][d] = kg.st[0][d];
    }
    p->kg = k2;
  }
  p->swapped = swap ? 1 : 0;
  p->batched = bl.empty() ? 0 : 1;
  p->bg = bg;
  if (swap)
    for (int d = 0; d < bg.D; ++d) {
      p->bg.st[0][d] = bg.st[1][d];
      p->bg.st[1][d] = bg.st[0][d];
    }
  p->bgc = bgc;
  p->P = bg.length();
  p->M = p->mg.length();
  p->N = p->ng.length();
  p->K = p->kg.length();

  bool ok;
  int64_t s;
  s = p->mg.ramp_step(0, ok); p->a_mfast = ok && (s == 1 || s == -1);
  s = p->ng.ramp_step(0, ok); p->b_nfast = ok && (s == 1 || s == -1);
  s = p->mg.ramp_step(1, ok); p->c_mfast = ok && (s == 1 || s == -1);
  if (!p->a_mfast) {
    // first non-singleton M axis unit-stride in A is enough for coalescing
    for (int d = 0; d < p->mg.D; ++d) {
      if (p->mg.len[d] == 1) continue;
      p->a_mfast = (p->mg.st[0][d] == 1 || p->mg.st[0][d] == -1);
      break;
    }
  }
  if (!p->b_nfast) {
    for (int d = 0; d < p->ng.D; ++d) {
      if (p->ng.len[d] == 1) continue;
      p->b_nfast = (p->ng.st[0][d] == 1 || p->ng.st[0][d] == -1);
      break;
    }
  }
  if (!p->c_mfast) {
    for (int d = 0; d < p->mg.D; ++d) {
      if (p->mg.len[d] == 1) continue;
      p->c_mfast = (p->mg.st[1][d] == 1 || p->mg.st[1][d] == -1);
      break;
    }
  }

  // select_path (src/planning/plan.jl:395-412), device thresholds.  A
  // batched plan runs the gather GEMM (or a tensor-core method) per entry.
  if (p->M == 0 || p->N == 0 || p->P == 0) {
    p->path = QS_PATH_EMPTY;
  } else if (p->K == 0) {
    p->path = QS_PATH_SCALE;
  } else if (p->batched) {
    p->path = QS_PATH_NEST;
  } else if ((p->M == 1 || p->N == 1) && p->K >= 32 && o.dot_mode != QS_MODE_NEVER) {
    p->path = QS_PATH_DOT;
  } else if (p->K == 1 && o.outer_mode != QS_MODE_NEVER) {
    p->path = QS_PATH_OUTER;
  } else {
    p->path = QS_PATH_NEST;
  }

  // Bounds are checked now and reported by qs_execute before any launch.
  p->bounds_ok_c = 1;
  p->bounds_ok_ab = 1;
  if (p->path != QS_PATH_EMPTY) {
    if (check_bounds(p, false) != QS_OK) {
      p->bounds_ok_c = 0;
    } else if (p->path != QS_PATH_SCALE && check_bounds(p, true) != QS_OK) {
      p->bounds_ok_ab = 0;
    }
  }
  set_error(QS_OK, "");
  return QS_OK;
}

}  // namespace qs

extern "C" size_t qs_last_error(char *buf, size_t n) {
  const std::string &m = qs::g_last.msg;
  if (buf && n > 0) {
    size_t k = m.size() < n - 1 ? m.size() : n - 1;
    std::memcpy(buf, m.data(), k);
    buf[k] = '\0';
  }
  return m.size();
}
