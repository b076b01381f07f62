// Internal declarations shared by the host planner (planner.cpp), the C ABI
// (api.cu) and the kernel translation units.
#pragma once

#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/qsgpu.h"

namespace qs {

// An NVTX range over a scope (plan, execute, group execute): visible in
// Nsight timelines, a no-op unless a profiler is attached.
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

constexpr int kMaxRank = 16;  // labels per M/N/K composite

// A grouped tensor axis: D dims enumerated by one zero-based coordinate,
// first dim fastest, with two stride maps (src/layout/axis_group.jl:5-23).
// Map 0/1 are (A, C) for M, (B, C) for N and (A, B) for K.
struct Group {
  int D = 0;
  int64_t len[kMaxRank] = {};
  int64_t st[2][kMaxRank] = {};
  int64_t label[kMaxRank] = {};
  int64_t length() const {
    int64_t q = 1;
    for (int d = 0; d < D; ++d) q *= len[d];
    return q;
  }
  // (lo, hi) of map p's offsets over the whole group; (0, -1) when empty.
  void offset_range(int p, int64_t &lo, int64_t &hi) const;
  // Step of map p when it is a single ramp (offset(q) = q*step), else
  // sets ok=false (src/layout/axis_group.jl:149-168).
  int64_t ramp_step(int p, bool &ok) const;
  // Mixed-radix offsets of coordinates [first, first+count) of map p
  // (src/layout/axis_group.jl:87-145).
  void fill_offsets(int p, int64_t first, int64_t count, int64_t *out) const;
};

struct Status {
  int code = QS_OK;
  std::string msg;
};

// Thread-local last error used by qs_last_error.
void set_error(int code, const std::string &msg);
int fail(int code, const std::string &msg);

inline bool is_complex(int t) { return t == QS_C32 || t == QS_C64; }
inline bool is_double(int t) { return t == QS_F64 || t == QS_C64; }
inline int elsize(int t) {
  switch (t) {
    case QS_F32: return 4;
    case QS_F64: return 8;
    case QS_C32: return 8;
    case QS_C64: return 16;
  }
  return 0;
}
const char *eltype_name(int t);

// Device workspace of a plan: offset tables and packed panels.  Owned by the
// plan, allocated at plan time, freed by qs_plan_destroy.
struct Workspace {
  // offset tables, device int64: M maps (A, C), N maps (B, C), K maps (A, B)
  int64_t *offM[2] = {nullptr, nullptr};
  int64_t *offN[2] = {nullptr, nullptr};
  int64_t *offK[2] = {nullptr, nullptr};
  // batch labels: [A offsets | B offsets | C offsets], P each, or nullptr
  int64_t *offBatch = nullptr;
  // tensor-core paths: packed operand panels and per-row/col exponents
  void *panelA = nullptr;
  void *panelB = nullptr;
  int32_t *expA = nullptr;  // per packed row of A (Ozaki), or nullptr
  int32_t *expB = nullptr;
  unsigned long long *rowmax = nullptr;  // Ozaki: row maxima of A (Mp) then B (Np)
  int32_t *rperm[2] = {nullptr, nullptr};  // Ozaki pack row orders (A, B), or nullptr
  int32_t *status = nullptr;  // device status word (bounded waits)
  size_t bytes = 0;
  std::vector<void *> owned;         // every allocated block, for freeing
  std::vector<size_t> owned_bytes;   // and its size (for a qs_allocator)
};

struct TensorCoreGeom {
  // Padded problem in packed-panel units.
  int64_t Mp = 0, Np = 0, Kp = 0;  // padded rows of A/B panels and K
  int64_t mtiles = 0, ntiles = 0, kblocks = 0;
  int rows_per_elem_a = 1;  // 1m: 2 real rows per complex row of A
  int cols_per_elem_b = 1;  // planar: 2 real columns per complex column of B
  int cplx_layout = 0;      // 0 real, 1 = 1m (A "1e", B "1r"), 2 = planar (A "1r", B "1e")
  int kmul = 1;             // 1m: 2 real K per complex K
  int nslices = 0;          // Ozaki slices (or 2 planes hi/lo for bf16x3)
  int64_t plane_bytes_a = 0, plane_bytes_b = 0;
  int kseg = 0;             // K blocks per INT32-exact segment (Ozaki)
};

}  // namespace qs

struct qs_plan {
  // Operand roles after the optional swap: "A" feeds M, "B" feeds N.
  int TA = 0, TB = 0, TC = 0;
  int T = 0;  // compute type
  int conjA = 0, conjB = 0;  // effective conjugation (flag XOR op), per role
  int swapped = 0;
  void *Adata = nullptr, *Bdata = nullptr, *Cdata = nullptr;
  int64_t Alen = 0, Blen = 0, Clen = 0;
  int64_t Abase = 0, Bbase = 0, Cbase = 0;
  qs::Group mg, ng, kg;
  int64_t M = 0, N = 0, K = 0;
  // Batch labels (QS_PLAN_BATCH_LABELS): bg maps A and B (after the swap),
  // bgc maps C; P batch entries; batch_host = the uploaded offset table.
  int batched = 0;
  qs::Group bg, bgc;
  int64_t P = 1;
  std::vector<int64_t> batch_host;
  int path = QS_PATH_EMPTY;
  int method = QS_METHOD_NATIVE;
  int complex_mode = QS_CPLX_NONE;
  int ozaki_slices = 0;
  int bounds_ok_c = 1, bounds_ok_ab = 1;
  std::string bounds_msg;
  int host_only = 0;
  int device = 0;
  // Tensor-core kernels: bound of every barrier wait, and the failure-
  // detection hold (qs_plan_set_wait_limit).
  uint64_t wait_ns = 2000000000ull;
  int hold_loads = 0;
  qs_plan_options opts{};
  // Workspace allocator (qs_plan_options.allocator), copied; has_alloc == 0
  // means the library's stream-ordered pool.  last_stream is the stream of
  // the last qs_execute (a freed block's work may still run there); grouped
  // plans may also have run on a group's side streams.
  qs_allocator alloc{};
  int has_alloc = 0;
  void *last_stream = nullptr;
  int grouped = 0;
  int executed = 0;
  // cudaEvent_t recorded on the setup stream after the plan's uploads and
  // clears; executes wait for it until it has completed (then it is freed).
  void *ready = nullptr;
  // Per-path launch flags chosen at plan time.
  int a_mfast = 0;  // A's M map is unit-stride (gather along M)
  int b_nfast = 0;  // B's N map is unit-stride (gather along N)
  int c_mfast = 0;  // C's M map is unit-stride
  int native_shape = 0;  // gather-GEMM tile shape (direct_shape numbering)
  qs::TensorCoreGeom tc;
  qs::Workspace ws;
  // CTA-pair Ozaki kernel: tensor maps (CUtensorMap bytes) of the A and B
  // panels, made once the panels exist; oz_pair_maps == 0 -> one-SM kernel.
  int oz_pair_maps = 0;
  unsigned char oz_tmap[256] = {};
  // Instrumentation (qs_plan_profile): cudaEvent_t handles, kProfStages+1
  // per recorded execute.
  static constexpr int kProfExec = 256, kProfStages = 5;
  int prof_on = 0, prof_nexec = 0, prof_nstages = 0;
  std::vector<void *> prof_events;
  // CUDA-graph replay (QS_PLAN_CUDA_GRAPH): graph, instance, capture stream
  // and the alpha/beta baked into it.
  void *graph = nullptr, *graph_exec = nullptr, *cap_stream = nullptr;
  double gal[2] = {0, 0}, gbe[2] = {0, 0};
  int capturing = 0;
};

namespace qs {
// Plan-time device copies and clears, on a private non-blocking stream of the
// calling thread (never the legacy default stream, which would serialize
// planning with work in flight on other streams); both wait for completion.
// Return a cudaError_t code.
int setup_copy(void *dst, const void *src, size_t bytes, int to_device);
int setup_zero(void *dst, size_t bytes);
// Plan workspace: stream-ordered allocation on the setup stream (from the
// device's default pool, which keeps freed memory cached), so planning
// never waits for kernels in flight.  Freeing synchronizes the device first:
// the plan's last executes may still be running on any stream.
int device_alloc(void **p, size_t bytes);
// Plan-time device work without host waits: pageable uploads, clears, and
// the ready event that orders a plan's executes after them.
void *plan_setup_stream();
int setup_upload(void *dst, const void *src, size_t bytes);
int setup_zero_async(void *dst, size_t bytes);
void plan_mark_ready(qs_plan *p);
void plan_wait_ready(qs_plan *p, void *stream);  // stream wait (host wait under capture)
void plan_sync_ready(qs_plan *p);                    // host wait
// The built-in device arena (arena.cu): recognized so that plan workspace
// reusing reclaimed memory waits on `stream` instead of the host.
bool is_arena_allocator(const qs_allocator *a);
int arena_alloc_ordered(void *ctx, size_t bytes, void **out, void *stream);
// A block of plan workspace from the plan's allocator (or the pool), recorded
// in p->ws for freeing; QS_ENOMEM (with the message set) on failure.
int plan_alloc(qs_plan *p, void **out, size_t bytes);
void device_free_all(std::vector<void *> &ptrs);

// planner.cpp
// Shape, eltype and op checks of one view (QS_EINVAL with a message).
int validate_view(const qs_view *v, const char *name);
int plan_host(qs_plan *p, const qs_view *C, const qs_view *A,
              const int64_t *indA, const qs_view *B, const int64_t *indB,
              const int64_t *indC, const qs_plan_options *opts);
int check_bounds(const qs_plan *p, bool reads_ab);
}  // namespace qs
