// Grouped execution (qs_group_*): many independent plans, e.g. the charge
// sectors of one block-sparse contraction, executed with one launch per
// stage and kernel class instead of one launch sequence per plan.
//
// Classes: the gather GEMM per compute type (one grouped launch each), the
// tensor-core paths per GEMM kernel (Ozaki with 6 or 7 slices, the
// per-product INT8 kernel, split-BF16x3: prep/pack/GEMM/fixup launches
// each).  Dot, outer and scale plans, and plans whose alpha is zero, run
// their own qs_execute.  Tables are rebuilt only when alpha/beta change.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <sstream>
#include <vector>

#include "kernels.h"
#include "qs_internal.h"
#include "tc.h"

using namespace qs;

struct qs_group {
  int mode = QS_GROUP_PERSISTENT;
  std::vector<qs_plan *> plans;
  // Persistent mode: the classes and the plans that run on their own.
  NativeGroup native[4 * kNativeShapes];  // by compute type QS_F32..QS_C64 x native shape
  TcGroup tc[TC_NCLASS];
  std::vector<int> single;
  bool built = false;
  std::vector<double> alpha, beta;  // values the tables/graph hold
  int launches = 0;
  // Persistent mode: side streams that run the classes concurrently (fork
  // and join through events on the caller's stream).
  static constexpr int kSide = 4;
  cudaStream_t side[kSide] = {};
  cudaEvent_t fork = nullptr, join[kSide] = {};
  // Stream-ordered release of the device tables: `last_use` is recorded on
  // the caller's stream after every execute; frees go on `rel` after it.
  cudaStream_t rel = nullptr;
  cudaEvent_t last_use = nullptr;
  bool used_since_build = false;
  // Graph mode.
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  cudaStream_t cap_stream = nullptr;
  int capturing = 0;
};

namespace {

int gfail(cudaError_t e, const char *what) {
  std::ostringstream s;
  s << "CUDA error in " << what << ": " << cudaGetErrorString(e);
  return fail(QS_ECUDA, s.str());
}

void release_tables(qs_group *g) {
  if (g->rel && g->used_since_build) cudaStreamWaitEvent(g->rel, g->last_use, 0);
  for (auto &c : g->native) {
    if (c.dev) cudaFreeAsync(c.dev, g->rel);
    c = NativeGroup{};
  }
  for (auto &c : g->tc) {
    tc_group_release(c, g->rel);
    c = TcGroup{};
  }
  g->single.clear();
  g->built = false;
  g->used_since_build = false;
}

int ensure_release_stream(qs_group *g) {
  if (g->rel) return QS_OK;
  cudaError_t e = cudaStreamCreateWithFlags(&g->rel, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->last_use, cudaEventDisableTiming);
  return e == cudaSuccess ? QS_OK : gfail(e, "stream/event creation");
}

// After launches on `st` that read the current tables.
int mark_use(qs_group *g, cudaStream_t st) {
  cudaError_t e = cudaEventRecord(g->last_use, st);
  if (e != cudaSuccess) return gfail(e, "cudaEventRecord");
  g->used_since_build = true;
  return QS_OK;
}

void release_graph(qs_group *g) {
  if (g->graph_exec) cudaGraphExecDestroy(g->graph_exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  g->graph_exec = nullptr;
  g->graph = nullptr;
}

// Sort key of the persistent launches' longest-first order: per-tile work.
int64_t plan_cost(const qs_plan *p) {
  if (p->method == QS_METHOD_NATIVE) return p->K;
  return p->tc.kblocks;
}

// Class membership, device tables and their upload for the given scalars.
int build_tables(qs_group *g, const double *alpha, const double *beta, cudaStream_t st) {
  int rc0 = ensure_release_stream(g);
  if (rc0) return rc0;
  release_tables(g);
  const int n = (int)g->plans.size();
  std::vector<int> bcase(n);
  std::vector<std::vector<int>> nat(4 * kNativeShapes), tcm(TC_NCLASS);
  for (int i = 0; i < n; ++i) {
    qs_plan *p = g->plans[i];
    const int acase = scalar_case(p->T, alpha + 2 * i);
    bcase[i] = scalar_case(p->T, beta + 2 * i);
    if (p->path == QS_PATH_EMPTY) continue;
    if (acase == 0 || p->path != QS_PATH_NEST) {
      g->single.push_back(i);
    } else if (p->method == QS_METHOD_NATIVE) {
      // The 32x32 tile exists to fill the GPU with one small problem; in a
      // group the other problems fill it, so the N-based shape is used unless
      // the plan asked for 32x32 itself.
      const int sh = p->opts.native_tile == 0
                         ? native_shape_for(p->T, p->TA, p->TB, p->M, p->N, p->K, 0, true)
                         : p->native_shape;
      nat[kNativeShapes * (p->T - QS_F32) + sh].push_back(i);
    } else {
      tcm[tc_group_class(p)].push_back(i);
    }
  }
  auto by_cost = [&](std::vector<int> &v) {
    std::stable_sort(v.begin(), v.end(), [&](int a, int b) {
      return plan_cost(g->plans[a]) > plan_cost(g->plans[b]);
    });
  };
  int rc;
  for (int t = 0; t < 4 * kNativeShapes; ++t) {
    if (nat[t].empty()) continue;
    by_cost(nat[t]);
    NativeGroup &c = g->native[t];
    c.T = QS_F32 + t / kNativeShapes;
    c.shape = t % kNativeShapes;
    std::vector<Operands> ops;
    for (int i : nat[t]) {
      c.plans.push_back(g->plans[i]);
      c.idx.push_back(i);
      ops.push_back(make_operands(g->plans[i]));
    }
    if ((rc = native_group_build(c, ops.data(), alpha, beta, bcase.data()))) return rc;
    cudaError_t e = cudaMallocAsync(&c.dev, c.image.size(), st);
    if (e != cudaSuccess) {
      cudaGetLastError();
      c.dev = nullptr;
      return fail(QS_ENOMEM, "device allocation of a grouped launch's tables failed");
    }
    c.dev_bytes = c.image.size();
    e = cudaMemcpyAsync(c.dev, c.image.data(), c.image.size(), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return gfail(e, "cudaMemcpyAsync (grouped launch tables)");
  }
  for (int k = 0; k < TC_NCLASS; ++k) {
    if (tcm[k].empty()) continue;
    by_cost(tcm[k]);
    TcGroup &c = g->tc[k];
    c.cls = k;
    for (int i : tcm[k]) {
      c.plans.push_back(g->plans[i]);
      c.idx.push_back(i);
    }
    if ((rc = tc_group_build(c, alpha, beta, bcase.data()))) return rc;
    if ((rc = tc_group_upload(c, st))) return rc;
  }
  g->alpha.assign(alpha, alpha + 2 * n);
  g->beta.assign(beta, beta + 2 * n);
  g->built = true;
  return QS_OK;
}

// qs_execute of one member plan: its launches go straight onto the group's
// stream (a plan-level graph or event profile would not be part of the
// group's sequence or graph).
int execute_member(qs_plan *p, const double *alpha, const double *beta, cudaStream_t st) {
  const int cap = p->capturing, prof = p->prof_on;
  p->capturing = 1;
  p->prof_on = 0;
  int rc = qs_execute(p, alpha, beta, (void *)st);
  p->capturing = cap;
  p->prof_on = prof;
  return rc;
}

int ensure_side_streams(qs_group *g) {
  if (g->fork) return QS_OK;
  cudaError_t e = cudaEventCreateWithFlags(&g->fork, cudaEventDisableTiming);
  for (int i = 0; e == cudaSuccess && i < qs_group::kSide; ++i) {
    e = cudaStreamCreateWithFlags(&g->side[i], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->join[i], cudaEventDisableTiming);
  }
  return e == cudaSuccess ? QS_OK : gfail(e, "stream/event creation");
}

// Singles on the caller's stream, then each class on a side stream (the
// classes are independent: the plans write disjoint C), joined back.
int launch_persistent(qs_group *g, const double *alpha, const double *beta, cudaStream_t st) {
  int launches = 0;
  for (int i : g->single) {
    const int64_t before = qs_launch_count();
    int rc = execute_member(g->plans[i], alpha + 2 * i, beta + 2 * i, st);
    if (rc) return rc;
    launches += (int)(qs_launch_count() - before);
  }
  int rc = ensure_side_streams(g);
  if (rc) return rc;
  cudaError_t e = cudaEventRecord(g->fork, st);
  if (e != cudaSuccess) return gfail(e, "cudaEventRecord");
  bool used[qs_group::kSide] = {};
  int next = 0;
  auto pick = [&]() -> cudaStream_t {
    const int i = next++ % qs_group::kSide;
    if (!used[i]) {
      cudaStreamWaitEvent(g->side[i], g->fork, 0);
      used[i] = true;
    }
    return g->side[i];
  };
  // Tensor-core classes first: they are the longest.
  for (auto &c : g->tc) {
    if (c.plans.empty()) continue;
    if ((rc = tc_group_launch(c, pick(), &launches))) return rc;
  }
  for (auto &c : g->native) {
    if (c.plans.empty()) continue;
    e = native_group_launch(c, pick());
    if (e != cudaSuccess) return gfail(e, "grouped gather-GEMM launch");
    count_launches(1);
    ++launches;
  }
  for (int i = 0; i < qs_group::kSide; ++i) {
    if (!used[i]) continue;
    e = cudaEventRecord(g->join[i], g->side[i]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, g->join[i], 0);
    if (e != cudaSuccess) return gfail(e, "stream join");
  }
  g->launches = launches;
  return QS_OK;
}

int launch_sequential(qs_group *g, const double *alpha, const double *beta, cudaStream_t st) {
  const int64_t before = qs_launch_count();
  for (size_t i = 0; i < g->plans.size(); ++i) {
    int rc = execute_member(g->plans[i], alpha + 2 * i, beta + 2 * i, st);
    if (rc) return rc;
  }
  g->launches = (int)(qs_launch_count() - before);
  return QS_OK;
}

int launch(qs_group *g, const double *alpha, const double *beta, cudaStream_t st) {
  if (g->mode & QS_GROUP_SEQUENTIAL) return launch_sequential(g, alpha, beta, st);
  return launch_persistent(g, alpha, beta, st);
}

bool same_scalars(const qs_group *g, const double *alpha, const double *beta) {
  const size_t n = g->plans.size() * 2;
  return g->alpha.size() == n && std::equal(alpha, alpha + n, g->alpha.begin()) &&
         std::equal(beta, beta + n, g->beta.begin());
}

}  // namespace

extern "C" {

int qs_group_create(int32_t n, qs_plan *const *plans, int32_t mode, qs_group **out) {
  if (!out) return fail(QS_EINVAL, "ArgumentError: group output pointer is NULL");
  *out = nullptr;
  if (n < 0 || (n > 0 && !plans)) return fail(QS_EINVAL, "ArgumentError: invalid grouped arguments");
  if (mode & ~(QS_GROUP_SEQUENTIAL | QS_GROUP_GRAPH))
    return fail(QS_EINVAL, "ArgumentError: unknown group mode");
  for (int i = 0; i < n; ++i) {
    if (!plans[i]) return fail(QS_EINVAL, "ArgumentError: plan is NULL");
    if (plans[i]->host_only)
      return fail(QS_EINVAL, "ArgumentError: a host-only plan has no device workspace to execute");
    if (plans[i]->batched)
      return fail(QS_ENOTSUP, "ArgumentError: a plan with batch labels cannot join a group");
    for (int j = 0; j < i; ++j)
      if (plans[j] == plans[i]) return fail(QS_EINVAL, "ArgumentError: a plan appears twice in a group");
  }
  qs_group *g = new (std::nothrow) qs_group();
  if (!g) return fail(QS_ENOMEM, "host allocation failed");
  g->mode = mode;
  g->plans.assign(plans, plans + n);
  for (int i = 0; i < n; ++i) {
    plans[i]->grouped = 1;      // frees of its workspace wait for the device
    plan_sync_ready(plans[i]);  // group launches and captures need its setup done
  }
  *out = g;
  return QS_OK;
}

int qs_group_execute(qs_group *g, const double *alpha, const double *beta, void *stream) {
  qs::NvtxRange nvtx("qs_group_execute");
  if (!g) return fail(QS_EINVAL, "ArgumentError: group is NULL");
  const int n = (int)g->plans.size();
  if (n == 0) return QS_OK;
  if (!alpha || !beta) return fail(QS_EINVAL, "ArgumentError: alpha/beta is NULL");
  // Every check of every plan before anything is enqueued.
  for (int i = 0; i < n; ++i) {
    qs_plan *p = g->plans[i];
    if (!is_complex(p->T) && (alpha[2 * i + 1] != 0.0 || beta[2 * i + 1] != 0.0))
      return fail(QS_EINVAL, "InexactError: a complex alpha/beta does not convert to the real compute type");
    if (p->path == QS_PATH_EMPTY) continue;
    const bool scale_only = scalar_case(p->T, alpha + 2 * i) == 0 || p->path == QS_PATH_SCALE;
    int rc = check_bounds(p, !scale_only);
    if (rc) return rc;
  }
  cudaStream_t st = (cudaStream_t)stream;
  cudaSetDevice(g->plans[0]->device);
  const bool same = same_scalars(g, alpha, beta);
  const bool graph = (g->mode & QS_GROUP_GRAPH) != 0;
  if (!graph) {
    if (!(g->mode & QS_GROUP_SEQUENTIAL) && (!g->built || !same)) {
      int rc = build_tables(g, alpha, beta, st);
      if (rc) return rc;
    }
    int rc = launch(g, alpha, beta, st);
    if (rc) return rc;
    return g->built ? mark_use(g, st) : QS_OK;
  }
  if (!g->graph_exec || !same) {
    release_graph(g);
    cudaError_t e;
    if (!g->cap_stream) {
      e = cudaStreamCreateWithFlags(&g->cap_stream, cudaStreamNonBlocking);
      if (e != cudaSuccess) return gfail(e, "cudaStreamCreateWithFlags");
    }
    if (!(g->mode & QS_GROUP_SEQUENTIAL)) {
      // Tables are uploaded outside the capture, on the capture stream, and
      // complete before it begins.
      int rc = build_tables(g, alpha, beta, g->cap_stream);
      if (rc) return rc;
      e = cudaStreamSynchronize(g->cap_stream);
      if (e != cudaSuccess) return gfail(e, "cudaStreamSynchronize");
    }
    e = cudaStreamBeginCapture(g->cap_stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return gfail(e, "cudaStreamBeginCapture");
    int rc = launch(g, alpha, beta, g->cap_stream);
    cudaGraph_t gr = nullptr;
    e = cudaStreamEndCapture(g->cap_stream, &gr);
    if (rc) {
      if (gr) cudaGraphDestroy(gr);
      return rc;
    }
    if (e != cudaSuccess) return gfail(e, "cudaStreamEndCapture");
    cudaGraphExec_t x;
    e = cudaGraphInstantiate(&x, gr, 0);
    if (e != cudaSuccess) {
      cudaGraphDestroy(gr);
      return gfail(e, "cudaGraphInstantiate");
    }
    g->graph = gr;
    g->graph_exec = x;
    g->alpha.assign(alpha, alpha + 2 * n);
    g->beta.assign(beta, beta + 2 * n);
  }
  cudaError_t e = cudaGraphLaunch(g->graph_exec, st);
  if (e != cudaSuccess) return gfail(e, "cudaGraphLaunch");
  return g->built ? mark_use(g, st) : QS_OK;
}

int qs_group_get_info(const qs_group *g, qs_group_info *info) {
  if (!g || !info) return fail(QS_EINVAL, "ArgumentError: group/info is NULL");
  std::memset(info, 0, sizeof(*info));
  info->nplans = (int32_t)g->plans.size();
  info->launches = g->launches;
  info->single_plans = (int32_t)g->single.size();
  for (const auto &c : g->native) {
    if (c.plans.empty()) continue;
    info->native_plans += (int32_t)c.plans.size();
    info->classes += 1;
    info->table_bytes += (int64_t)c.dev_bytes;
  }
  for (const auto &c : g->tc) {
    if (c.plans.empty()) continue;
    info->tc_plans += (int32_t)c.plans.size();
    info->classes += 1;
    info->tiles += c.tiles;
    info->table_bytes += (int64_t)c.dev_bytes;
  }
  return QS_OK;
}

int qs_group_destroy(qs_group *g) {
  if (!g) return QS_OK;
  if (!g->plans.empty()) cudaSetDevice(g->plans[0]->device);
  release_graph(g);
  release_tables(g);
  if (g->rel) cudaStreamDestroy(g->rel);  // its frees still run after the device work
  if (g->last_use) cudaEventDestroy(g->last_use);
  if (g->cap_stream) cudaStreamDestroy(g->cap_stream);
  for (int i = 0; i < qs_group::kSide; ++i) {
    if (g->side[i]) cudaStreamDestroy(g->side[i]);
    if (g->join[i]) cudaEventDestroy(g->join[i]);
  }
  if (g->fork) cudaEventDestroy(g->fork);
  delete g;
  return QS_OK;
}

int qs_execute_grouped(int32_t n, qs_plan *const *plans, const double *alpha, const double *beta,
                       void *stream) {
  qs_group *g = nullptr;
  int rc = qs_group_create(n, plans, QS_GROUP_PERSISTENT, &g);
  if (rc) return rc;
  rc = qs_group_execute(g, alpha, beta, stream);
  if (rc == QS_OK) {
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) rc = gfail(e, "cudaStreamSynchronize");
  }
  qs_group_destroy(g);
  return rc;
}

}  // extern "C"
