/*
 * qsgpu.h — C ABI of the B200 contraction engine (libqsgpu.so).
 *
 * Computes C[indC] = alpha * sum_K op(A)[indA] * op(B)[indB] + beta * C[indC]
 * over strided ("block-scatter") operands that live in device memory, with
 * the semantics of QuasiStrided.jl's engine:
 *
 *   plan_contract  src/planning/plan.jl:115-133   -> qs_plan_contract
 *   execute!       src/execution/execute.jl:11   -> qs_execute
 *   contract!      src/execution/execute.jl:84   -> qs_contract
 *   release!       src/execution/workspace.jl:118 -> qs_plan_destroy
 *   QuasiStridedBackend(; accumulator)            -> qs_plan_options.accumulator
 *     src/integrations/tensoroperations.jl:24-32
 *   TO.tensorcontract! label mapping              -> qs_contraction_labels
 *     src/integrations/tensoroperations.jl:40-47
 *   TO.tensoradd! / TO.tensortrace! (forwarded to StridedNative there)
 *     src/integrations/tensoroperations.jl:91-107  -> qs_tensoradd_trace
 *   TensorOperations allocators for the workspace -> qs_plan_options.allocator,
 *     src/execution/workspace.jl:98-123              qs_arena_* (BufferAllocator)
 *
 * Conventions
 *  - Every operand is a qs_view: a parent allocation (`data`, `length`
 *    elements) plus a StridedView-style (size, strides, offset, op) window
 *    into it; strides are in elements and may be zero or negative
 *    (StridedViews.jl's StridedView fields).
 *  - Labels are one int64 per axis, as in the reference (`indA`, `indB`,
 *    `indC`): a label in A and B but not C is contracted (K); a label in C
 *    and exactly one of A/B is free (M or N).  Any other pattern is QS_EINVAL.
 *  - Scalars (alpha, beta) are passed as two doubles {re, im}; for a real
 *    compute type a nonzero imaginary part is QS_EINVAL (Julia's
 *    `convert(T, alpha)` throws InexactError).
 *  - Every validation happens before anything is written: plan-time errors
 *    come from qs_plan_contract, out-of-bounds operands from qs_execute before
 *    any launch (the reference checks spans with checked_span_bounds,
 *    src/layout/tiles.jl:123-140, before a block is written;
 *    test/execution/test_execute.jl:57-70).
 *  - No C++ exception crosses this boundary.  The message of the last error
 *    on the calling thread is available from qs_last_error.
 *  - A plan borrows the operands' device memory and owns its device
 *    workspace (offset tables, packed panels).  One stream per execute; a plan
 *    must not be executed concurrently with itself (src/planning/plan.jl:12).
 */
#ifndef QSGPU_H
#define QSGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The Julia/Python hosts map them to the reference's exception
 * types: EINVAL -> ArgumentError, EDIM -> DimensionMismatch,
 * EBOUNDS -> BoundsError. */
enum {
  QS_OK = 0,
  QS_EINVAL = 1,   /* ArgumentError: labels, eltypes, conjugated C, aliasing */
  QS_EDIM = 2,     /* DimensionMismatch: a label's axis lengths differ */
  QS_EBOUNDS = 3,  /* BoundsError: a view reaches outside its parent */
  QS_ENOMEM = 4,   /* device allocation failed (plan time only) */
  QS_ETIMEOUT = 5, /* a device-side bounded wait gave up (status flag) */
  QS_ECUDA = 6,    /* a CUDA runtime call failed */
  QS_ENOTSUP = 7   /* requested method/kernel not available for this plan */
};

/* Element types: QuasiStrided's SUPPORTED_ELTYPES (src/planning/plan.jl:264). */
enum { QS_F32 = 0, QS_F64 = 1, QS_C32 = 2, QS_C64 = 3 };

/* StridedView.op (src/planning/plan.jl:176-186). */
enum { QS_OP_IDENTITY = 0, QS_OP_CONJ = 1, QS_OP_TRANSPOSE = 2, QS_OP_ADJOINT = 3 };

/* accumulator keyword: nothing / Float32 / Float64 (src/planning/plan.jl:278-285). */
enum { QS_ACC_NONE = 0, QS_ACC_F32 = 1, QS_ACC_F64 = 2 };

/* GEMM method for the nest path.  AUTO follows the autotuner's choice. */
enum {
  QS_METHOD_AUTO = 0,
  QS_METHOD_NATIVE = 1,   /* gather GEMM without tensor-core splitting: real Float64
                             operands on the FP64 tensor cores (DMMA, mma.sync f64),
                             other types as a SIMT FMA kernel */
  QS_METHOD_OZAKI_I8 = 2, /* FP64 (6-7 digits) or FP32 (4 digits) as INT8 slices on tcgen05 kind::i8 */
  QS_METHOD_BF16X3 = 3    /* FP32 as split-BF16 x3 on tcgen05 kind::f16 */
};

/* Path modes (src/planning/plan.jl:60-64 PathModes). */
enum { QS_MODE_AUTO = 0, QS_MODE_NEVER = 1, QS_MODE_ALWAYS = 2 };

/* Execution paths (src/execution/paths.jl). */
enum {
  QS_PATH_EMPTY = 0,
  QS_PATH_SCALE = 1,
  QS_PATH_DOT = 2,
  QS_PATH_OUTER = 3,
  QS_PATH_NEST = 4
};

/* Complex formulations on the real tensor-core paths. */
enum { QS_CPLX_NONE = 0, QS_CPLX_PLANAR = 1, QS_CPLX_1M = 2 };

/* Plan flags. */
enum {
  QS_PLAN_HOST_ONLY = 1, /* plan on the host only: no device workspace; the
                            plan can be inspected but not executed */
  QS_PLAN_PER_PRODUCT_GEMM = 2, /* Ozaki: one slice product per pipeline stage
                                   (the simpler kernel) instead of grouped
                                   diagonals with resident slice tiles */
  QS_PLAN_CUDA_GRAPH = 4, /* qs_execute captures the plan's launches into a
                             CUDA graph once (again when alpha/beta change)
                             and replays it on later calls */
  QS_PLAN_OZ_SINGLE_SM = 16, /* Ozaki with 6 or 7 slices: the one-SM GEMM kernel
                                instead of the CTA-pair (cta_group::2) kernel */
  QS_PLAN_BATCH_LABELS = 8 /* accept labels present in A, B and C (which the
                              reference rejects, src/planning/labels.jl:48-54)
                              as batch labels: C[b,...] = alpha * sum_K
                              A[b,...] B[b,...] + beta * C[b,...] for every b */
};

typedef struct qs_view {
  void *data;             /* device pointer to element 0 of the parent */
  int64_t length;         /* parent length in elements */
  int64_t offset;         /* element offset of the view's first element */
  const int64_t *size;    /* [ndim] */
  const int64_t *strides; /* [ndim], in elements */
  int32_t ndim;
  int32_t eltype; /* QS_F32 .. QS_C64 */
  int32_t op;     /* QS_OP_* */
  int32_t reserved;
} qs_view;

/* A device allocator for plan workspace: TensorOperations' `allocator`
 * argument of plan_contract (src/planning/plan.jl:115-133), whose
 * ContractWorkspace takes its panels with tensoralloc and hands them back with
 * tensorfree! in reverse order (src/execution/workspace.jl:98-123).
 *   alloc: at least `bytes` bytes of device memory on the current device,
 *          aligned to 256 bytes, free for work enqueued after the call on any
 *          stream; NULL when it has none (the plan then fails with QS_ENOMEM).
 *   free:  hands a block back; a plan's blocks come back in the reverse order
 *          of allocation.  `stream` is the stream of the plan's last execute
 *          (NULL: the legacy default stream); work on it that used the block
 *          may still be running, so an allocator that reuses the block orders
 *          the reuse after that work (the built-in qs_arena does).
 * The plan keeps a copy of this struct; `ctx` must outlive the plan. */
typedef struct qs_allocator {
  void *ctx;
  void *(*alloc)(void *ctx, size_t bytes);
  void (*free)(void *ctx, void *ptr, size_t bytes, void *stream);
} qs_allocator;

typedef struct qs_plan_options {
  int32_t conjA;       /* conjugate A's elements (XOR with A's op) */
  int32_t conjB;       /* conjugate B's elements (XOR with B's op) */
  int32_t accumulator; /* QS_ACC_* */
  int32_t method;      /* QS_METHOD_* */
  int64_t m_block;     /* blocking hints (src/planning/blocking.jl:9-20): */
  int64_t k_block;     /* 0 = default; values < 0 are QS_EINVAL.  On the */
  int64_t n_block;     /* device they only bound the K segment length.   */
  int32_t dot_mode;    /* QS_MODE_* */
  int32_t outer_mode;  /* QS_MODE_* */
  int32_t unpacked_b_mode; /* QS_MODE_* (read-B-in-place skinny path) */
  int32_t ozaki_slices;    /* 0 = chosen from K for 1e-13; else 2..10 */
  int32_t complex_mode;    /* QS_CPLX_*; 0 = default for the method */
  int32_t flags;           /* QS_PLAN_* */
  int32_t native_tile;     /* native-method tile: 0 = by M and N; SIMT gather kernel
                              1 = 64x64, 2 = 128x32, 3 = 256x16, 4 = 32x32 (real
                              compute types); DMMA kernel (real Float64 A and B)
                              5 = 128x128, 6 = 128x64, 7 = 64x64, 8 = 128x32,
                              9 = 256x16, 10 = 128x128 with 16 warps (the
                              autotuner's knob) */
  const qs_allocator *allocator; /* plan workspace from here; NULL = the library's
                                    stream-ordered pool (DefaultAllocator) */
} qs_plan_options;

typedef struct qs_plan_info {
  int32_t path;         /* QS_PATH_* */
  int32_t method;       /* QS_METHOD_* actually used by the nest path */
  int32_t compute_type; /* QS_F32 .. QS_C64 */
  int32_t swapped;      /* 1 when B takes the M role */
  int32_t conjA;        /* effective conjugation of the M-side operand */
  int32_t conjB;        /* effective conjugation of the N-side operand */
  int32_t ozaki_slices;
  int32_t complex_mode;
  int64_t m_length, n_length, k_length;
  int32_t m_rank, n_rank, k_rank;
  int32_t bounds_ok; /* 0 when qs_execute would return QS_EBOUNDS */
  int64_t m_labels[16], n_labels[16], k_labels[16]; /* group label order */
  int64_t workspace_bytes;
  int32_t stride_class;  /* bit 0: A's M map unit-stride, bit 1: B's N map,
                            bit 2: C's M map (the autotuner's stride class) */
  int32_t native_tile;   /* native-method tile in use (1..10 as in the options) */
  int32_t batch_rank;    /* batch labels (QS_PLAN_BATCH_LABELS), 0 without */
  int64_t batch_length;  /* product of their extents (1 without) */
  int64_t batch_labels[16];
} qs_plan_info;

typedef struct qs_plan qs_plan;

/* plan_contract (src/planning/plan.jl:115-133).  indA/indB/indC hold
 * A->ndim, B->ndim, C->ndim labels.  opts may be NULL (all defaults). */
int qs_plan_contract(qs_plan **plan, const qs_view *C, const qs_view *A,
                     const int64_t *indA, const qs_view *B,
                     const int64_t *indB, const int64_t *indC,
                     const qs_plan_options *opts);

/* execute! (src/execution/execute.jl:11-20): alpha/beta are {re, im}.
 * stream is a cudaStream_t (NULL = legacy default stream).  Asynchronous:
 * returns once the work is enqueued. */
int qs_execute(qs_plan *plan, const double *alpha, const double *beta,
               void *stream);

/* contract! (src/execution/execute.jl:84-95): plan, execute, release in one
 * call.  The plan's workspace is freed stream-ordered after the work: with
 * the library's pool the call waits for `stream`; with opts->allocator it
 * returns once the work is enqueued and hands the workspace back with
 * `stream` (the allocator orders its reuse, as the qs_arena does). */
int qs_contract(const qs_view *C, const double *alpha, const qs_view *A,
                const int64_t *indA, const qs_view *B, const int64_t *indB,
                const double *beta, const int64_t *indC,
                const qs_plan_options *opts, void *stream);

/* release! (src/execution/workspace.jl:118-123) plus freeing the plan. */
int qs_plan_destroy(qs_plan *plan);

/* Inspection of a plan (path, groups, method) for hosts and tests. */
int qs_plan_get_info(const qs_plan *plan, qs_plan_info *info);

/* Re-point a plan at new operand storage of identical layout (same parent
 * lengths, offsets): src/planning/plan.jl:48-56 rebuilds a plan with new
 * storages the same way.  Used by the serving loop to reuse plans. */
int qs_plan_rebind(qs_plan *plan, void *A_data, void *B_data, void *C_data);

/* TO.tensorcontract! label mapping (src/integrations/tensoroperations.jl:40-47):
 * pA = (pA_out[NoA], pA_in[Nk]), pB = (pB_in[Nk], pB_out[NoB]),
 * pAB = (pAB_1 ++ pAB_2)[NoA+NoB], all 1-based as in Julia.  Writes
 * indA[NoA+Nk], indB[Nk+NoB], indC[NoA+NoB]. */
int qs_contraction_labels(int32_t NoA, int32_t Nk, int32_t NoB,
                          const int64_t *pA_lin, const int64_t *pB_lin,
                          const int64_t *pAB_lin, int64_t *indA,
                          int64_t *indB, int64_t *indC);

/* Grouped execution of many independent plans: the block-sparse
 * contraction step of a symmetric tensor network, where each charge sector
 * is one plan.  No counterpart in the reference, whose engine runs one plan
 * per contract! call (src/execution/execute.jl:84-95); each plan's result
 * is that of qs_execute on it.
 *
 * Modes:
 *   QS_GROUP_PERSISTENT  plans sharing a kernel class (compute type for the
 *                        gather GEMM; method and slice count for the tensor-
 *                        core paths) run as ONE launch per stage: a grouped
 *                        pack, a persistent GEMM whose CTAs walk the tiles
 *                        of a device problem table, one fixup.  Dot, outer
 *                        and scale plans run as their own launches.
 *   QS_GROUP_SEQUENTIAL  one qs_execute per plan, in order (the baseline).
 *   QS_GROUP_GRAPH       (flag) the launches of an execute are captured into
 *                        a CUDA graph once and replayed; alpha/beta changes
 *                        re-capture.
 * The plans must not share C with each other, must not be executed on their
 * own while the group is in use, and stay owned by the caller (destroy the
 * group first).  All bounds are checked for every plan before any launch. */
typedef struct qs_group qs_group;
enum {
  QS_GROUP_PERSISTENT = 0,
  QS_GROUP_SEQUENTIAL = 1,
  QS_GROUP_GRAPH = 2
};

typedef struct qs_group_info {
  int32_t nplans;
  int32_t launches;      /* kernels per execute (last execute) */
  int32_t native_plans;  /* plans in grouped gather-GEMM launches */
  int32_t tc_plans;      /* plans in grouped tensor-core launches */
  int32_t single_plans;  /* plans run as their own launches */
  int32_t classes;       /* grouped launch classes in use */
  int64_t tiles;         /* tensor-core tiles per execute */
  int64_t table_bytes;   /* device bytes of the problem tables */
} qs_group_info;

int qs_group_create(int32_t n, qs_plan *const *plans, int32_t mode, qs_group **out);
/* alpha/beta: {re, im} per plan (2*n doubles each).  Enqueued on `stream`. */
int qs_group_execute(qs_group *g, const double *alpha, const double *beta, void *stream);
int qs_group_get_info(const qs_group *g, qs_group_info *info);
int qs_group_destroy(qs_group *g);

/* One-shot grouped execute: create (QS_GROUP_PERSISTENT), execute, wait for
 * the stream, destroy. */
int qs_execute_grouped(int32_t n, qs_plan *const *plans, const double *alpha,
                       const double *beta, void *stream);

/* TO.tensoradd! / TO.tensortrace! on the device, which the reference forwards
 * to StridedNative on the host (src/integrations/tensoroperations.jl:90-107):
 *   C[indC] = alpha * sum over traced labels of op(A)[indA] + beta * C[indC]
 * Every label of indC appears exactly once in indA (a permutation: tensoradd!);
 * every other label of indA appears exactly twice (a traced pair:
 * tensortrace!).  conjA is XORed with A's op; a conjugated C is rejected.
 * beta == 0 never reads C, alpha == 0 never reads A; bounds are checked
 * before any launch.  One kernel on `stream`; allocates nothing. */
int qs_tensoradd_trace(const qs_view *C, const double *alpha, const qs_view *A,
                       const int64_t *indA, int32_t conjA, const double *beta,
                       const int64_t *indC, void *stream);

/* contract! without any device allocation.  No counterpart in the reference:
 * it is for callers that cannot allocate device memory when they contract,
 * e.g. a serving loop where cudaMalloc/cudaFree would synchronize the device
 * and stall other in-flight work, or a host whose memory pool forbids raw
 * allocations.  It plans on the host and runs the gather kernels with their
 * M/N/K offset tables in one fixed-size file-scope device array, so it needs
 * 2*(M+N+K) <= 524288 (QS_EINVAL otherwise) and does not use the
 * tensor-core paths.  All calls share that array: calls that overlap on the
 * GPU race.  The first call on a device looks the array up and should come
 * before any stream capture on that device.  Arguments as qs_contract;
 * returns once the work is enqueued on `stream`. */
int qs_contract_noalloc(const qs_view *C, const double *alpha, const qs_view *A,
                        const int64_t *indA, const qs_view *B,
                        const int64_t *indB, const double *beta,
                        const int64_t *indC, const qs_plan_options *opts,
                        void *stream);

/* Instrumentation.  With profiling enabled, qs_execute records CUDA events
 * around each of its launches (pack A, pack B, GEMM, fixup for the
 * tensor-core paths; the single kernel otherwise) for up to 256 executes.
 * qs_plan_stage_times synchronizes on those events and returns, per stage,
 * the summed milliseconds, the stage count and the number of executes
 * recorded; it then clears the record. */
int qs_plan_profile(qs_plan *plan, int32_t enable);
int qs_plan_stage_times(qs_plan *plan, double *stage_ms, int32_t max_stages,
                        int32_t *nstages, int32_t *nexec);

/* Device status word of a plan's tensor-core kernels: synchronizes `stream`,
 * returns QS_ETIMEOUT (and clears the word) if a bounded wait gave up since
 * the last check, else QS_OK. */
int qs_plan_check_status(qs_plan *plan, void *stream);

/* Failure detection (no counterpart in the reference, whose engine has no
 * device waits).  Every barrier wait of the plan's tensor-core kernels gives
 * up after `limit_ns` (0: the default, 2 s); the kernel then stops without
 * writing C, waits (with the same bound) for the copies and MMAs it already
 * issued, releases its tensor memory and returns, and qs_plan_check_status
 * reports QS_ETIMEOUT; the GPU and the plan stay usable.  `hold_loads` != 0
 * makes the GEMM's producers issue no operand copies at all, so the first
 * wait for an operand tile runs out with nothing in flight: a way for tests
 * to exercise that error path without a fault.  A captured graph of the plan
 * (QS_PLAN_CUDA_GRAPH) is re-captured at the next execute.  Limits above
 * 60 s are QS_EINVAL. */
int qs_plan_set_wait_limit(qs_plan *plan, uint64_t limit_ns, int32_t hold_loads);

/* Device arena: the device counterpart of TensorOperations' BufferAllocator
 * (the allocators plan_contract accepts; checkpoint/reset bracket every
 * TO.tensorcontract!, src/integrations/tensoroperations.jl:84-86).  A bump
 * allocator over one device buffer: O(1) allocation with no cudaMalloc and
 * no synchronization, blocks handed back LIFO, everything above a checkpoint
 * reclaimed by a reset.  Memory that a free or a reset hands back is reused
 * only after the work enqueued before it on the given stream is done (the
 * allocation that reuses it waits on an event).  Thread-safe.
 *   create:     base == NULL allocates `bytes` with cudaMalloc on the current
 *               device (freed by destroy); otherwise the arena serves the
 *               caller's device memory [base, base+bytes) (a CuArray, a torch
 *               tensor), which must outlive it.
 *   allocator:  the qs_allocator to put in qs_plan_options.allocator.
 *   alloc/free: tensoralloc / tensorfree! of intermediates (256-byte aligned;
 *               QS_ENOMEM when the arena is full).  free of the top block pops
 *               it (and any freed blocks under it); of another block marks it;
 *               of a block a reset already reclaimed does nothing.
 *   checkpoint: allocator_checkpoint! (the current top, in bytes).
 *   reset:      allocator_reset!: drops every block above `checkpoint`; `stream`
 *               is where the work that used them was enqueued. */
typedef struct qs_arena qs_arena;
int qs_arena_create(qs_arena **arena, void *base, size_t bytes);
int qs_arena_destroy(qs_arena *arena);
const qs_allocator *qs_arena_allocator(qs_arena *arena);
int qs_arena_alloc(qs_arena *arena, size_t bytes, void **out);
int qs_arena_free(qs_arena *arena, void *ptr, size_t bytes, void *stream);
size_t qs_arena_checkpoint(qs_arena *arena);
int qs_arena_reset(qs_arena *arena, size_t checkpoint, void *stream);
/* used = current top, peak = highest top since create, capacity = bytes,
 * waits = allocations that had to wait for reclaimed memory's work. */
int qs_arena_get_info(qs_arena *arena, size_t *used, size_t *peak, size_t *capacity, int64_t *waits);

/* Number of device kernels this library has launched in this process
 * (instrumentation: benchmarks difference it around a timed region). */
int64_t qs_launch_count(void);

/* Message of the last error on this thread; returns its full length. */
size_t qs_last_error(char *buf, size_t n);

/* Library version string. */
const char *qs_version(void);

#ifdef __cplusplus
}
#endif

#endif /* QSGPU_H */
