// Device arena: the device counterpart of TensorOperations' BufferAllocator.
//
// The reference takes a plan's packed panels and panel of C from the
// TensorOperations allocator (src/execution/workspace.jl:98-123) and brackets
// every TO.tensorcontract! with allocator_checkpoint!/allocator_reset!
// (src/integrations/tensoroperations.jl:84-86).  On the device the point of
// an arena is that planning then needs no cudaMalloc (each of which is a host
// round trip on the setup stream) and a served network's workspace and
// intermediates stay inside one fixed buffer.
//
// A bump allocator: `top` grows by 256-byte-aligned blocks kept on a stack.
// Freeing the top block pops it (and any blocks under it already freed);
// freeing another block only marks it; a reset drops every block above the
// checkpoint.  The device may still be using memory that a free or a reset
// hands back, so each of those records an event on the stream that used it;
// the first later allocation that overlaps memory handed out before the
// event waits for it (a host wait on an event that is normally complete).
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <sstream>
#include <vector>

#include "qs_internal.h"

namespace {

constexpr size_t kAlign = 256;

struct Block {
  size_t off, bytes;
  bool freed;
};

}  // namespace

struct qs_arena {
  char *base = nullptr;
  size_t cap = 0;
  size_t top = 0;
  size_t peak = 0;
  // End of the memory handed out since the fences were last waited for: an
  // allocation below it reuses memory the device may still be using.
  size_t dirty = 0;
  int64_t waits = 0;
  int device = 0;  // -1: no CUDA device (bookkeeping only, nothing to order)
  bool owns = false;
  std::vector<Block> blocks;
  std::vector<cudaEvent_t> fences;  // recorded, not yet waited for
  std::vector<cudaEvent_t> spare;   // waited for, reusable
  qs_allocator iface{};
  std::mutex mu;
};

namespace {

using qs::fail;

// Moves fences whose work is done to the spare list; true when none is left
// (caller holds the lock, current device set).
bool prune_fences(qs_arena *a) {
  size_t keep = 0;
  for (cudaEvent_t ev : a->fences) {
    if (cudaEventQuery(ev) == cudaSuccess) {
      a->spare.push_back(ev);
    } else {
      cudaGetLastError();  // cudaErrorNotReady is not a failure
      a->fences[keep++] = ev;
    }
  }
  a->fences.resize(keep);
  return keep == 0;
}

// Records a fence on `stream` (caller holds the lock, current device set).
int add_fence(qs_arena *a, void *stream) {
  if (a->device < 0) return QS_OK;
  prune_fences(a);
  cudaEvent_t ev = nullptr;
  if (!a->spare.empty()) {
    ev = a->spare.back();
    a->spare.pop_back();
  } else {
    cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess) {
      cudaGetLastError();
      // Without an event, order the reuse after all device work.
      cudaDeviceSynchronize();
      return QS_OK;
    }
  }
  cudaError_t e = cudaEventRecord(ev, (cudaStream_t)stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    a->spare.push_back(ev);
    cudaDeviceSynchronize();
    return QS_OK;
  }
  a->fences.push_back(ev);
  return QS_OK;
}

// Waits for every recorded fence (caller holds the lock).
int wait_fences(qs_arena *a) {
  cudaError_t first = cudaSuccess;
  for (cudaEvent_t ev : a->fences) {
    cudaError_t e = cudaEventSynchronize(ev);
    if (e != cudaSuccess && first == cudaSuccess) first = e;
    a->spare.push_back(ev);
  }
  if (!a->fences.empty()) ++a->waits;
  a->fences.clear();
  if (first != cudaSuccess) {
    std::ostringstream m;
    m << "CUDA error while waiting for reclaimed arena memory: " << cudaGetErrorString(first);
    return fail(QS_ECUDA, m.str());
  }
  return QS_OK;
}

struct DeviceGuard {
  int prev = 0;
  bool on = false;
  explicit DeviceGuard(int dev) : on(dev >= 0) {
    if (!on) return;
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    if (!on) return;
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != prev) cudaSetDevice(prev);
  }
};

// `order` == nullptr: reuse of reclaimed memory waits on the host (memory
// usable by any later work).  Otherwise the stream `*order` waits instead,
// and only work ordered after that stream may use the block.
int arena_alloc(qs_arena *a, size_t bytes, void **out, const cudaStream_t *order = nullptr) {
  *out = nullptr;
  std::lock_guard<std::mutex> lk(a->mu);
  const size_t n = std::max<size_t>(kAlign, (bytes + kAlign - 1) / kAlign * kAlign);
  if (bytes > a->cap || n > a->cap - a->top) {
    std::ostringstream m;
    m << "device arena exhausted: " << bytes << " bytes requested, " << (a->cap - a->top) << " of "
      << a->cap << " free";
    return fail(QS_ENOMEM, m.str());
  }
  const size_t off = a->top;
  if (off < a->dirty && !a->fences.empty()) {
    DeviceGuard g(a->device);
    if (prune_fences(a)) {
      a->dirty = off;
    } else if (order) {
      for (cudaEvent_t ev : a->fences) {
        cudaError_t e = cudaStreamWaitEvent(*order, ev, 0);
        if (e != cudaSuccess) {
          std::ostringstream m;
          m << "cudaStreamWaitEvent on reclaimed arena memory: " << cudaGetErrorString(e);
          return fail(QS_ECUDA, m.str());
        }
      }
      ++a->waits;
    } else {
      int rc = wait_fences(a);
      if (rc) return rc;
      a->dirty = off;
    }
  }
  a->blocks.push_back(Block{off, n, false});
  a->top = off + n;
  a->peak = std::max(a->peak, a->top);
  a->dirty = std::max(a->dirty, a->top);
  *out = a->base + off;
  return QS_OK;
}

int arena_free(qs_arena *a, void *ptr, size_t bytes, void *stream) {
  (void)bytes;
  if (!ptr) return QS_OK;
  char *p = static_cast<char *>(ptr);
  if (p < a->base || p >= a->base + a->cap)
    return fail(QS_EINVAL, "ArgumentError: pointer does not belong to this device arena");
  const size_t off = (size_t)(p - a->base);
  std::lock_guard<std::mutex> lk(a->mu);
  auto it = std::find_if(a->blocks.begin(), a->blocks.end(), [&](const Block &b) { return b.off == off; });
  if (it == a->blocks.end()) return QS_OK;  // already reclaimed by a reset
  it->freed = true;
  while (!a->blocks.empty() && a->blocks.back().freed) {
    a->top = a->blocks.back().off;
    a->blocks.pop_back();
  }
  // The fence goes on this free's stream whether the block popped now or
  // only got marked: a marked block is popped later by a free on another
  // stream, whose fence says nothing about the work on this one.
  DeviceGuard g(a->device);
  return add_fence(a, stream);
}

void *iface_alloc(void *ctx, size_t bytes) {
  void *p = nullptr;
  return arena_alloc(static_cast<qs_arena *>(ctx), bytes, &p) == QS_OK ? p : nullptr;
}

void iface_free(void *ctx, void *ptr, size_t bytes, void *stream) {
  arena_free(static_cast<qs_arena *>(ctx), ptr, bytes, stream);
}

}  // namespace

namespace qs {
bool is_arena_allocator(const qs_allocator *al) { return al && al->alloc == iface_alloc; }

int arena_alloc_ordered(void *ctx, size_t bytes, void **out, void *stream) {
  const cudaStream_t st = (cudaStream_t)stream;
  return arena_alloc(static_cast<qs_arena *>(ctx), bytes, out, &st);
}
}  // namespace qs

extern "C" {

int qs_arena_create(qs_arena **out, void *base, size_t bytes) {
  if (!out) return fail(QS_EINVAL, "ArgumentError: arena output pointer is NULL");
  *out = nullptr;
  if (base && (reinterpret_cast<uintptr_t>(base) % kAlign))
    return fail(QS_EINVAL, "ArgumentError: arena base must be 256-byte aligned");
  qs_arena *a = new (std::nothrow) qs_arena();
  if (!a) return fail(QS_ENOMEM, "host allocation failed");
  cudaError_t e = cudaGetDevice(&a->device);
  if (e != cudaSuccess) {
    // No device: only an arena over the caller's memory, as bookkeeping.
    cudaGetLastError();
    if (!base) {
      delete a;
      return fail(QS_ECUDA, std::string("device arena: ") + cudaGetErrorString(e));
    }
    a->device = -1;
    a->base = static_cast<char *>(base);
  } else if (base) {
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, base) != cudaSuccess ||
        (pa.type != cudaMemoryTypeDevice && pa.type != cudaMemoryTypeManaged)) {
      cudaGetLastError();
      delete a;
      return fail(QS_EINVAL, "ArgumentError: the arena's base is not device memory");
    }
    a->device = pa.device;
    a->base = static_cast<char *>(base);
  } else if (bytes) {
    void *p = nullptr;
    e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      delete a;
      std::ostringstream m;
      m << "device arena of " << bytes << " bytes: " << cudaGetErrorString(e);
      return fail(QS_ENOMEM, m.str());
    }
    a->base = static_cast<char *>(p);
    a->owns = true;
  }
  a->cap = bytes;
  a->iface.ctx = a;
  a->iface.alloc = iface_alloc;
  a->iface.free = iface_free;
  *out = a;
  return QS_OK;
}

int qs_arena_destroy(qs_arena *a) {
  if (!a) return QS_OK;
  if (a->device >= 0) {
    std::lock_guard<std::mutex> lk(a->mu);
    DeviceGuard g(a->device);
    wait_fences(a);
    for (cudaEvent_t ev : a->spare) cudaEventDestroy(ev);
    a->spare.clear();
    if (a->owns && a->base) {
      cudaDeviceSynchronize();  // nothing may still use the buffer
      cudaFree(a->base);
    }
  }
  delete a;
  return QS_OK;
}

const qs_allocator *qs_arena_allocator(qs_arena *a) { return a ? &a->iface : nullptr; }

int qs_arena_alloc(qs_arena *a, size_t bytes, void **out) {
  if (!a || !out) return fail(QS_EINVAL, "ArgumentError: NULL argument");
  return arena_alloc(a, bytes, out);
}

int qs_arena_free(qs_arena *a, void *ptr, size_t bytes, void *stream) {
  if (!a) return fail(QS_EINVAL, "ArgumentError: arena is NULL");
  return arena_free(a, ptr, bytes, stream);
}

size_t qs_arena_checkpoint(qs_arena *a) {
  if (!a) return 0;
  std::lock_guard<std::mutex> lk(a->mu);
  return a->top;
}

int qs_arena_reset(qs_arena *a, size_t checkpoint, void *stream) {
  if (!a) return fail(QS_EINVAL, "ArgumentError: arena is NULL");
  std::lock_guard<std::mutex> lk(a->mu);
  if (checkpoint > a->top) return fail(QS_EINVAL, "ArgumentError: checkpoint lies above the arena's top");
  if (checkpoint == a->top) return QS_OK;
  for (auto it = a->blocks.rbegin(); it != a->blocks.rend(); ++it)
    if (it->off < checkpoint) {
      if (it->off + it->bytes > checkpoint)
        return fail(QS_EINVAL, "ArgumentError: checkpoint is not a value qs_arena_checkpoint returned");
      break;
    }
  while (!a->blocks.empty() && a->blocks.back().off >= checkpoint) a->blocks.pop_back();
  a->top = checkpoint;
  DeviceGuard g(a->device);
  return add_fence(a, stream);
}

int qs_arena_get_info(qs_arena *a, size_t *used, size_t *peak, size_t *capacity, int64_t *waits) {
  if (!a) return fail(QS_EINVAL, "ArgumentError: arena is NULL");
  std::lock_guard<std::mutex> lk(a->mu);
  if (used) *used = a->top;
  if (peak) *peak = a->peak;
  if (capacity) *capacity = a->cap;
  if (waits) *waits = a->waits;
  return QS_OK;
}

}  // extern "C"
