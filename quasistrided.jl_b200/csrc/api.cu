// The C ABI (include/qsgpu.h): plan creation, execution and destruction.
//
//   qs_plan_contract <- plan_contract / planned (src/planning/plan.jl:115-262)
//   qs_execute       <- execute! (src/execution/execute.jl:11-20)
//   qs_contract      <- contract! (src/execution/execute.jl:84-95)
//   qs_plan_destroy  <- release! (src/execution/workspace.jl:118-123)
//
// All validation happens on the host before anything is written; kernels
// are launched asynchronously on the caller's stream.  No exception crosses
// the boundary.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <sstream>
#include <vector>

#include "kernels.h"
#include "qs_internal.h"
#include "tc.h"

using namespace qs;

#include <atomic>

namespace qs {
static std::atomic<int64_t> g_launches{0};
void count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

static cudaStream_t setup_stream(cudaError_t *err) {
  thread_local cudaStream_t s = nullptr;
  thread_local int dev = -1;
  int cur = 0;
  cudaGetDevice(&cur);
  if (!s || dev != cur) {
    *err = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    dev = cur;
  }
  return s;
}

void *plan_setup_stream() {
  cudaError_t e = cudaSuccess;
  return (void *)setup_stream(&e);
}

int setup_upload(void *dst, const void *src, size_t bytes) {
  cudaError_t e = cudaSuccess;
  cudaStream_t s = setup_stream(&e);
  if (e != cudaSuccess) return (int)e;
  // From pageable memory the call returns once `src` is staged: no wait.
  return (int)cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
}

int setup_zero_async(void *dst, size_t bytes) {
  cudaError_t e = cudaSuccess;
  cudaStream_t s = setup_stream(&e);
  if (e != cudaSuccess) return (int)e;
  return (int)cudaMemsetAsync(dst, 0, bytes, s);
}

int setup_copy(void *dst, const void *src, size_t bytes, int to_device) {
  cudaError_t e = cudaSuccess;
  cudaStream_t s = setup_stream(&e);
  if (e != cudaSuccess) return (int)e;
  e = cudaMemcpyAsync(dst, src, bytes, to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return (int)e;
}

int device_alloc(void **p, size_t bytes) {
  cudaError_t e = cudaSuccess;
  cudaStream_t s = setup_stream(&e);
  if (e != cudaSuccess) return (int)e;
  thread_local int pool_dev = -1;
  int cur = 0;
  cudaGetDevice(&cur);
  if (pool_dev != cur) {
    // Keep freed pool memory mapped instead of returning it at every sync.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, cur) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    pool_dev = cur;
  }
  // Stream-ordered: the plan's ready event orders every later use.
  return (int)cudaMallocAsync(p, bytes, s);
}

void device_free_all(std::vector<void *> &ptrs) {
  if (ptrs.empty()) return;
  cudaError_t e = cudaSuccess;
  cudaStream_t s = setup_stream(&e);
  cudaDeviceSynchronize();
  for (void *q : ptrs) cudaFreeAsync(q, s);
  cudaStreamSynchronize(s);
  ptrs.clear();
}

int plan_alloc(qs_plan *p, void **out, size_t bytes) {
  *out = nullptr;
  if (p->has_alloc) {
    if (is_arena_allocator(&p->alloc)) {
      // Reuse of reclaimed arena memory waits on the setup stream, not the host.
      int rc = arena_alloc_ordered(p->alloc.ctx, bytes, out, plan_setup_stream());
      if (rc) {
        *out = nullptr;
        return rc;
      }
    } else {
      *out = p->alloc.alloc(p->alloc.ctx, bytes);
    }
    if (!*out) {
      std::ostringstream s;
      s << "the plan's allocator has no " << bytes << " bytes of device memory";
      return fail(QS_ENOMEM, s.str());
    }
  } else {
    cudaError_t e = (cudaError_t)device_alloc(out, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      *out = nullptr;
      std::ostringstream s;
      s << "device allocation of " << bytes << " bytes failed: " << cudaGetErrorString(e);
      return fail(QS_ENOMEM, s.str());
    }
  }
  p->ws.owned.push_back(*out);
  p->ws.owned_bytes.push_back(bytes);
  p->ws.bytes += bytes;
  return QS_OK;
}

void plan_mark_ready(qs_plan *p) {
  cudaError_t e = cudaSuccess;
  cudaStream_t s = setup_stream(&e);
  cudaEvent_t ev = nullptr;
  if (e == cudaSuccess && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess &&
      cudaEventRecord(ev, s) == cudaSuccess) {
    p->ready = (void *)ev;
    return;
  }
  cudaGetLastError();
  if (ev) cudaEventDestroy(ev);
  cudaStreamSynchronize(s);  // no event: finish the setup now
}

void plan_sync_ready(qs_plan *p) {
  if (!p->ready) return;
  cudaEventSynchronize((cudaEvent_t)p->ready);
  cudaEventDestroy((cudaEvent_t)p->ready);
  p->ready = nullptr;
}

void plan_wait_ready(qs_plan *p, void *stream) {
  if (!p->ready) return;
  cudaStream_t st = (cudaStream_t)stream;
  cudaEvent_t ev = (cudaEvent_t)p->ready;
  if (cudaEventQuery(ev) == cudaSuccess) {
    cudaEventDestroy(ev);
    p->ready = nullptr;
    return;
  }
  cudaGetLastError();  // cudaErrorNotReady is not a failure
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
    // A capture cannot wait on an event recorded outside it: finish now.
    cudaGetLastError();
    plan_sync_ready(p);
    return;
  }
  cudaStreamWaitEvent(st, ev, 0);
}

int setup_zero(void *dst, size_t bytes) {
  cudaError_t e = cudaSuccess;
  cudaStream_t s = setup_stream(&e);
  if (e != cudaSuccess) return (int)e;
  e = cudaMemsetAsync(dst, 0, bytes, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return (int)e;
}
}  // namespace qs

namespace qs {
Operands make_operands(const qs_plan *p) {
  Operands op;
  op.A = p->Adata;
  op.B = p->Bdata;
  op.C = p->Cdata;
  op.Abase = p->Abase;
  op.Bbase = p->Bbase;
  op.Cbase = p->Cbase;
  op.TA = p->TA;
  op.TB = p->TB;
  op.TC = p->TC;
  op.conjA = p->conjA;
  op.conjB = p->conjB;
  op.offMA = p->ws.offM[0];
  op.offMC = p->ws.offM[1];
  op.offNB = p->ws.offN[0];
  op.offNC = p->ws.offN[1];
  op.offKA = p->ws.offK[0];
  op.offKB = p->ws.offK[1];
  op.M = p->M;
  op.N = p->N;
  op.K = p->K;
  op.offBatch = p->ws.offBatch;
  op.P = p->batched ? p->P : 1;
  return op;
}

int scalar_case(int T, const double *v) {
  // Zero/One/general after conversion to the compute type.
  double re = v[0], im = is_complex(T) ? v[1] : 0.0;
  if (!is_double(T)) {
    re = (double)(float)re;
    im = (double)(float)im;
  }
  if (re == 0.0 && im == 0.0) return 0;
  if (re == 1.0 && im == 0.0) return 1;
  return 2;
}
}  // namespace qs

namespace {

int cuda_fail(cudaError_t e, const char *what) {
  std::ostringstream s;
  s << "CUDA error in " << what << ": " << cudaGetErrorString(e);
  return fail(QS_ECUDA, s.str());
}

void free_workspace(qs_plan *p) {
  if (p->has_alloc) {
    // Back to the caller's allocator in reverse order (release!,
    // src/execution/workspace.jl:118-123).  A grouped plan's last work may
    // be on a group's side streams, which the allocator cannot see: wait.
    if (p->grouped) {
      cudaDeviceSynchronize();
    } else if (!p->executed) {
      cudaError_t e = cudaSuccess;
      cudaStreamSynchronize(setup_stream(&e));  // plan-time uploads may be in flight
    }
    for (size_t i = p->ws.owned.size(); i-- > 0;)
      p->alloc.free(p->alloc.ctx, p->ws.owned[i], p->ws.owned_bytes[i], p->grouped ? nullptr : p->last_stream);
    p->ws.owned.clear();
  } else {
    device_free_all(p->ws.owned);
  }
  p->ws = Workspace{};
}

int ws_alloc(qs_plan *p, void **out, size_t bytes) {
  *out = nullptr;
  if (bytes == 0) return QS_OK;
  return plan_alloc(p, out, bytes);
}

// The M, N and K offset tables (two maps each) in one block and one copy.
int upload_offsets(qs_plan *p) {
  const Group *gs[3] = {&p->mg, &p->ng, &p->kg};
  int64_t **dst[3] = {p->ws.offM, p->ws.offN, p->ws.offK};
  size_t n[3], total = 0;
  for (int i = 0; i < 3; ++i) {
    const int64_t Q = gs[i]->length();
    n[i] = (size_t)(Q > 0 ? Q : 1);
    total += 2 * n[i];
  }
  const size_t nb = p->batched ? (size_t)p->P : 0;
  total += 3 * nb;
  std::vector<int64_t> h(total, 0);
  size_t at = 0;
  for (int i = 0; i < 3; ++i) {
    const int64_t Q = gs[i]->length();
    if (Q > 0) {
      gs[i]->fill_offsets(0, 0, Q, h.data() + at);
      gs[i]->fill_offsets(1, 0, Q, h.data() + at + n[i]);
    }
    at += 2 * n[i];
  }
  if (nb) {
    // [A | B | C] offsets of every batch entry, first batch label fastest.
    p->bg.fill_offsets(0, 0, (int64_t)nb, h.data() + at);
    p->bg.fill_offsets(1, 0, (int64_t)nb, h.data() + at + nb);
    p->bgc.fill_offsets(0, 0, (int64_t)nb, h.data() + at + 2 * nb);
    p->batch_host.assign(h.begin() + at, h.begin() + at + 3 * nb);
  }
  void *d;
  int rc = ws_alloc(p, &d, total * sizeof(int64_t));
  if (rc) return rc;
  cudaError_t e = (cudaError_t)setup_upload(d, h.data(), total * sizeof(int64_t));
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync (offset tables)");
  at = 0;
  for (int i = 0; i < 3; ++i) {
    dst[i][0] = (int64_t *)d + at;
    dst[i][1] = (int64_t *)d + at + n[i];
    at += 2 * n[i];
  }
  p->ws.offBatch = nb ? (int64_t *)d + at : nullptr;
  return QS_OK;
}

// Method for the nest path: the requested one if valid, else the
// autotuner's choice (tensor-core paths once the problem fills a tile).
int choose_method(qs_plan *p) {
  int want = p->opts.method;
  bool dbl = is_double(p->T);
  if (want == QS_METHOD_BF16X3 && dbl)
    return fail(QS_ENOTSUP, "ArgumentError: the split-BF16x3 method needs a Float32/ComplexF32 compute type");
  if (want < QS_METHOD_AUTO || want > QS_METHOD_BF16X3)
    return fail(QS_EINVAL, "ArgumentError: unknown method");
  if (want == QS_METHOD_AUTO) want = tc_auto_method(p);
  p->method = want;
  return QS_OK;
}

// The event slot of the next profiled execute (nullptr when profiling is off
// or the record is full).
cudaEvent_t *prof_slot(qs_plan *p) {
  if (!p->prof_on || p->prof_nexec >= qs_plan::kProfExec) return nullptr;
  return (cudaEvent_t *)p->prof_events.data() + (size_t)p->prof_nexec * (qs_plan::kProfStages + 1);
}

void destroy_graph(qs_plan *p) {
  if (p->graph_exec) cudaGraphExecDestroy((cudaGraphExec_t)p->graph_exec);
  if (p->graph) cudaGraphDestroy((cudaGraph_t)p->graph);
  p->graph_exec = nullptr;
  p->graph = nullptr;
}

}  // namespace

extern "C" int qs_execute(qs_plan *p, const double *alpha, const double *beta, void *stream);

namespace {

// execute! on a reused plan as a CUDA graph: the launches of one execute are
// captured on a private stream (capture of the legacy default stream is not
// allowed) and the instantiated graph is replayed on the caller's stream.
// alpha/beta are baked into the captured kernel parameters, so a change of
// either re-captures.
int execute_graph(qs_plan *p, const double *alpha, const double *beta, cudaStream_t st) {
  const bool same = p->graph_exec && p->gal[0] == alpha[0] && p->gal[1] == alpha[1] &&
                    p->gbe[0] == beta[0] && p->gbe[1] == beta[1];
  cudaError_t e;
  if (!same) {
    destroy_graph(p);
    if (!p->cap_stream) {
      cudaStream_t cs;
      e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
      if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreateWithFlags");
      p->cap_stream = (void *)cs;
    }
    cudaStream_t cs = (cudaStream_t)p->cap_stream;
    e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamBeginCapture");
    p->capturing = 1;
    const int prof = p->prof_on;
    p->prof_on = 0;  // no event records inside the graph
    int rc = qs_execute(p, alpha, beta, (void *)cs);
    p->prof_on = prof;
    p->capturing = 0;
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(cs, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    cudaGraphExec_t x;
    e = cudaGraphInstantiate(&x, g, 0);
    if (e != cudaSuccess) {
      cudaGraphDestroy(g);
      return cuda_fail(e, "cudaGraphInstantiate");
    }
    p->graph = (void *)g;
    p->graph_exec = (void *)x;
    p->gal[0] = alpha[0];
    p->gal[1] = alpha[1];
    p->gbe[0] = beta[0];
    p->gbe[1] = beta[1];
  }
  e = cudaGraphLaunch((cudaGraphExec_t)p->graph_exec, st);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGraphLaunch");
  return QS_OK;
}

}  // namespace

extern "C" {

size_t qs_last_error(char *buf, size_t n);  // defined below

int qs_plan_contract(qs_plan **out, const qs_view *C, const qs_view *A, const int64_t *indA,
                     const qs_view *B, const int64_t *indB, const int64_t *indC,
                     const qs_plan_options *opts) {
  qs::NvtxRange nvtx("qs_plan_contract");
  if (!out) return fail(QS_EINVAL, "ArgumentError: plan output pointer is NULL");
  *out = nullptr;
  qs_plan *p = new (std::nothrow) qs_plan();
  if (!p) return fail(QS_ENOMEM, "host allocation failed");
  int rc = plan_host(p, C, A, indA, B, indB, indC, opts);
  if (rc) {
    delete p;
    return rc;
  }
  if (p->opts.allocator) {
    const qs_allocator *al = p->opts.allocator;
    if (!al->alloc || !al->free) {
      delete p;
      return fail(QS_EINVAL, "ArgumentError: a qs_allocator needs both alloc and free");
    }
    p->alloc = *al;
    p->has_alloc = 1;
    p->opts.allocator = nullptr;  // the copy above is what the plan keeps
  }
  if (p->path == QS_PATH_NEST) {
    rc = choose_method(p);
    if (rc) {
      delete p;
      return rc;
    }
  } else {
    p->method = QS_METHOD_NATIVE;
  }
  const int nt = p->opts.native_tile;
  if (nt < 0 || nt > kNativeShapes) {
    delete p;
    return fail(QS_EINVAL, "ArgumentError: native_tile must be 0..10");
  }
  p->native_shape = native_shape_for(p->T, p->TA, p->TB, p->M, p->N, p->K, nt, false);
  if (!p->host_only) {
    cudaError_t e = cudaGetDevice(&p->device);
    if (e != cudaSuccess) {
      delete p;
      return cuda_fail(e, "cudaGetDevice");
    }
    if (p->path != QS_PATH_EMPTY) {
      if ((rc = upload_offsets(p))) {
        free_workspace(p);
        delete p;
        return rc;
      }
    }
    if (p->path == QS_PATH_NEST && p->method != QS_METHOD_NATIVE) {
      rc = tc_prepare(p);
      if (rc) {
        free_workspace(p);
        delete p;
        return rc;
      }
    }
    // The uploads and clears above are still in flight on the setup stream;
    // every execute waits for this event (qs_execute, groups, graphs).
    if (!p->ws.owned.empty()) plan_mark_ready(p);
  } else if (p->path == QS_PATH_NEST && p->method != QS_METHOD_NATIVE) {
    tc_geometry(p);
  }
  set_error(QS_OK, "");
  *out = p;
  return QS_OK;
}

int qs_execute(qs_plan *p, const double *alpha, const double *beta, void *stream) {
  qs::NvtxRange nvtx("qs_execute");
  if (!p) return fail(QS_EINVAL, "ArgumentError: plan is NULL");
  if (!alpha || !beta) return fail(QS_EINVAL, "ArgumentError: alpha/beta is NULL");
  if (p->host_only)
    return fail(QS_EINVAL, "ArgumentError: a host-only plan has no device workspace to execute");
  if (!is_complex(p->T) && (alpha[1] != 0.0 || beta[1] != 0.0))
    return fail(QS_EINVAL, "InexactError: a complex alpha/beta does not convert to the real compute type");
  if (!std::isfinite(alpha[0]) && std::isnan(alpha[0])) {
    // NaN alpha is a legal value: it propagates like the reference.
  }
  cudaStream_t st = (cudaStream_t)stream;
  if (!p->capturing) {
    plan_wait_ready(p, stream);
    p->last_stream = stream;
    p->executed = 1;
  }
  if ((p->opts.flags & QS_PLAN_CUDA_GRAPH) && !p->capturing) return execute_graph(p, alpha, beta, st);
  int acase = scalar_case(p->T, alpha);
  int bcase = scalar_case(p->T, beta);
  if (p->path == QS_PATH_EMPTY) return QS_OK;
  bool scale_only = (acase == 0) || p->path == QS_PATH_SCALE;
  int rc = check_bounds(p, !scale_only);
  if (rc) return rc;
  cudaSetDevice(p->device);
  Operands op = make_operands(p);
  cudaError_t e = cudaSuccess;
  cudaEvent_t *ev = prof_slot(p);
  if (scale_only) {
    if (bcase == 1) return QS_OK;  // C *= 1 is a no-op
    if (ev) cudaEventRecord(ev[0], st);
    e = launch_scale(p->T, op, beta, bcase, p->c_mfast, st);
    if (e != cudaSuccess) return cuda_fail(e, "scale kernel launch");
    if (ev) {
      cudaEventRecord(ev[1], st);
      p->prof_nstages = 1;
      ++p->prof_nexec;
    }
    count_launches(1);
    return QS_OK;
  }
  if (ev) cudaEventRecord(ev[0], st);
  switch (p->path) {
    case QS_PATH_DOT: e = launch_dot(p->T, op, alpha, beta, bcase, st); break;
    case QS_PATH_OUTER: e = launch_outer(p->T, op, alpha, beta, bcase, p->c_mfast, st); break;
    default:
      if (p->method == QS_METHOD_NATIVE) {
        e = launch_direct(p->T, op, alpha, beta, bcase, p->a_mfast, p->b_nfast, p->native_shape, st);
      } else {
        int rc2 = QS_OK;
        if (!p->batched) {
          rc2 = tc_execute(p, alpha, beta, bcase, st, ev);
        } else {
          // One tensor-core pass per batch entry, the operands rebased on
          // the host; the plan's panels are reused in stream order.
          const int64_t a0 = p->Abase, b0 = p->Bbase, c0 = p->Cbase, P = p->P;
          for (int64_t b = 0; b < P && rc2 == QS_OK; ++b) {
            p->Abase = a0 + p->batch_host[b];
            p->Bbase = b0 + p->batch_host[P + b];
            p->Cbase = c0 + p->batch_host[2 * P + b];
            rc2 = tc_execute(p, alpha, beta, bcase, st, b == 0 ? ev : nullptr);
          }
          p->Abase = a0;
          p->Bbase = b0;
          p->Cbase = c0;
        }
        if (rc2 == QS_OK && ev) ++p->prof_nexec;
        return rc2;
      }
  }
  if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
  if (ev) {
    cudaEventRecord(ev[1], st);
    p->prof_nstages = 1;
    ++p->prof_nexec;
  }
  count_launches(1);
  return QS_OK;
}

int qs_plan_profile(qs_plan *p, int32_t enable) {
  if (!p) return fail(QS_EINVAL, "ArgumentError: plan is NULL");
  if (p->host_only) return fail(QS_EINVAL, "ArgumentError: a host-only plan cannot be profiled");
  if (enable && p->prof_events.empty()) {
    const size_t n = (size_t)qs_plan::kProfExec * (qs_plan::kProfStages + 1);
    p->prof_events.resize(n, nullptr);
    for (size_t i = 0; i < n; ++i) {
      cudaEvent_t e;
      cudaError_t rc = cudaEventCreate(&e);
      if (rc != cudaSuccess) return cuda_fail(rc, "cudaEventCreate");
      p->prof_events[i] = (void *)e;
    }
  }
  p->prof_on = enable ? 1 : 0;
  p->prof_nexec = 0;
  return QS_OK;
}

int qs_plan_stage_times(qs_plan *p, double *stage_ms, int32_t max_stages, int32_t *nstages,
                        int32_t *nexec) {
  if (!p || !stage_ms || !nstages || !nexec) return fail(QS_EINVAL, "ArgumentError: NULL argument");
  const int ns = p->prof_nstages;
  for (int s = 0; s < max_stages; ++s) stage_ms[s] = 0.0;
  for (int x = 0; x < p->prof_nexec; ++x) {
    cudaEvent_t *ev = (cudaEvent_t *)p->prof_events.data() + (size_t)x * (qs_plan::kProfStages + 1);
    cudaError_t rc = cudaEventSynchronize(ev[ns]);
    if (rc != cudaSuccess) return cuda_fail(rc, "cudaEventSynchronize");
    for (int s = 0; s < ns && s < max_stages; ++s) {
      float ms = 0.f;
      rc = cudaEventElapsedTime(&ms, ev[s], ev[s + 1]);
      if (rc != cudaSuccess) return cuda_fail(rc, "cudaEventElapsedTime");
      stage_ms[s] += ms;
    }
  }
  *nstages = ns;
  *nexec = p->prof_nexec;
  p->prof_nexec = 0;
  return QS_OK;
}

int qs_plan_check_status(qs_plan *p, void *stream) {
  if (!p) return fail(QS_EINVAL, "ArgumentError: plan is NULL");
  if (p->host_only || !p->ws.status) return QS_OK;
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
  int32_t word = 0;
  e = (cudaError_t)setup_copy(&word, p->ws.status, sizeof(word), 0);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync (status)");
  if (word != 0) {
    setup_zero(p->ws.status, sizeof(int32_t));
    return fail(QS_ETIMEOUT, "a bounded device wait gave up (tensor-core kernel aborted)");
  }
  return QS_OK;
}

int qs_plan_set_wait_limit(qs_plan *p, uint64_t limit_ns, int32_t hold_loads) {
  if (!p) return fail(QS_EINVAL, "ArgumentError: plan is NULL");
  if (limit_ns > 60000000000ull)
    return fail(QS_EINVAL, "ArgumentError: a wait limit above 60 s is not a bound");
  p->wait_ns = limit_ns ? limit_ns : 2000000000ull;
  p->hold_loads = hold_loads ? 1 : 0;
  if (!p->host_only) destroy_graph(p);  // a captured graph holds the old arguments
  return QS_OK;
}

int qs_plan_destroy(qs_plan *p) {
  if (!p) return QS_OK;
  if (!p->host_only) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaSetDevice(p->device);
    for (void *e : p->prof_events)
      if (e) cudaEventDestroy((cudaEvent_t)e);
    p->prof_events.clear();
    destroy_graph(p);
    if (p->cap_stream) cudaStreamDestroy((cudaStream_t)p->cap_stream);
    p->cap_stream = nullptr;
    free_workspace(p);
    plan_sync_ready(p);
    cudaSetDevice(dev);
  }
  delete p;
  return QS_OK;
}

int qs_contract(const qs_view *C, const double *alpha, const qs_view *A, const int64_t *indA,
                const qs_view *B, const int64_t *indB, const double *beta, const int64_t *indC,
                const qs_plan_options *opts, void *stream) {
  qs::NvtxRange nvtx("qs_contract");
  qs_plan_options o{};
  if (opts) o = *opts;
  o.flags &= ~QS_PLAN_HOST_ONLY;
  qs_plan *p = nullptr;
  int rc = qs_plan_contract(&p, C, A, indA, B, indB, indC, &o);
  if (rc) return rc;
  rc = qs_execute(p, alpha, beta, stream);
  // The workspace is released once the enqueued work is done: by waiting
  // here, or, with a caller's allocator, by the allocator ordering its reuse
  // after `stream`.
  p->last_stream = stream;
  cudaError_t e = p->has_alloc ? cudaGetLastError() : cudaStreamSynchronize((cudaStream_t)stream);
  qs_plan_destroy(p);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
  return QS_OK;
}

int qs_plan_get_info(const qs_plan *p, qs_plan_info *info) {
  if (!p || !info) return fail(QS_EINVAL, "ArgumentError: NULL argument");
  std::memset(info, 0, sizeof(*info));
  info->path = p->path;
  info->method = p->method;
  info->compute_type = p->T;
  info->swapped = p->swapped;
  info->conjA = p->conjA;
  info->conjB = p->conjB;
  info->ozaki_slices = p->ozaki_slices;
  info->complex_mode = p->complex_mode;
  info->m_length = p->M;
  info->n_length = p->N;
  info->k_length = p->K;
  info->m_rank = p->mg.D;
  info->n_rank = p->ng.D;
  info->k_rank = p->kg.D;
  info->bounds_ok = p->bounds_ok_c && p->bounds_ok_ab;
  for (int d = 0; d < p->mg.D; ++d) info->m_labels[d] = p->mg.label[d];
  for (int d = 0; d < p->ng.D; ++d) info->n_labels[d] = p->ng.label[d];
  for (int d = 0; d < p->kg.D; ++d) info->k_labels[d] = p->kg.label[d];
  info->workspace_bytes = (int64_t)p->ws.bytes;
  info->stride_class = (p->a_mfast ? 1 : 0) | (p->b_nfast ? 2 : 0) | (p->c_mfast ? 4 : 0);
  info->native_tile = p->native_shape + 1;
  info->batch_rank = p->batched ? p->bg.D : 0;
  info->batch_length = p->batched ? p->P : 1;
  for (int d = 0; d < p->bg.D && d < 16; ++d) info->batch_labels[d] = p->bg.label[d];
  return QS_OK;
}

int qs_plan_rebind(qs_plan *p, void *A_data, void *B_data, void *C_data) {
  if (!p) return fail(QS_EINVAL, "ArgumentError: plan is NULL");
  void *a = p->swapped ? B_data : A_data;
  void *b = p->swapped ? A_data : B_data;
  if (a) p->Adata = a;
  if (b) p->Bdata = b;
  if (C_data) p->Cdata = C_data;
  destroy_graph(p);  // a captured graph holds the old pointers
  return QS_OK;
}

int qs_contraction_labels(int32_t NoA, int32_t Nk, int32_t NoB, const int64_t *pA_lin,
                          const int64_t *pB_lin, const int64_t *pAB_lin, int64_t *indA,
                          int64_t *indB, int64_t *indC) {
  // TO's pA/pB/pAB -> one label per axis (src/integrations/tensoroperations.jl:40-47):
  // 1:NoA for A's open axes (pA[1] order), NoA+1:NoA+NoB for B's open axes,
  // -1:-1:-Nk for the contracted pairs; indC = linearize(pAB).
  if (NoA < 0 || Nk < 0 || NoB < 0) return fail(QS_EINVAL, "ArgumentError: negative counts");
  int nA = NoA + Nk, nB = Nk + NoB;
  std::vector<int64_t> qA(nA), qB(nB);
  for (int i = 0; i < nA; ++i) {
    int64_t ax = pA_lin[i];
    if (ax < 1 || ax > nA) return fail(QS_EINVAL, "ArgumentError: invalid pA");
    qA[ax - 1] = i + 1;  // invperm
  }
  for (int i = 0; i < nB; ++i) {
    int64_t ax = pB_lin[i];
    if (ax < 1 || ax > nB) return fail(QS_EINVAL, "ArgumentError: invalid pB");
    qB[ax - 1] = i + 1;
  }
  for (int i = 0; i < nA; ++i) {
    int64_t s = qA[i];
    indA[i] = s <= NoA ? s : -(s - NoA);
  }
  for (int i = 0; i < nB; ++i) {
    int64_t s = qB[i];
    indB[i] = s <= Nk ? -s : NoA + (s - Nk);
  }
  for (int i = 0; i < NoA + NoB; ++i) indC[i] = pAB_lin[i];
  return QS_OK;
}

size_t qs_last_error(char *buf, size_t n);

const char *qs_version(void) { return "qsgpu 0.1.0 (sm_100a)"; }

int64_t qs_launch_count(void) { return qs::g_launches.load(std::memory_order_relaxed); }

}  // extern "C"
