"""Serving loop for contraction requests (continuous batching on one GPU).

Requests of mixed shapes and eltypes arrive over time.  Each loop iteration
(a *tick*):

1. collects completed ticks (their CUDA event has fired): results are already
   in pinned host buffers; budget, plans and buffers are released;
2. admits waiting requests in arrival order while their device bytes fit the
   HBM budget and a tick slot is free (requests that arrive while others are
   on the GPU are admitted as soon as slots and memory free up);
3. launches the admitted requests as one tick on its own stream: host->device
   copies, one grouped execute over all of them (``ContractGroup``: one
   launch per stage and kernel class), and the device->host copies of the
   results.

Host preparation is off that loop: with a backend that has ``prepare``, a
preparation thread stages each request as it arrives (device blocks, pinned
copies of host operands, its plan: reused from a cache and re-pointed with
``rebind``, so the steady state allocates no plan workspace), after charging
its bytes to the budget; the loop admits prepared requests only, in arrival
order.

Several ticks are in flight at once, so their work overlaps on the device.
Operands registered with ``put_resident`` stay on the device across requests
and count against the budget until removed.

The device work goes through a backend object (``DeviceBackend``); the
admission, ordering and accounting logic is backend-independent.  No
counterpart in the reference (a single-threaded library); this is the
serving front end of the engine's ``plan_contract``/``execute!``.
"""
from __future__ import annotations

import collections
import math
import threading
import time
from dataclasses import dataclass, field
from typing import Any, Optional, Sequence

import numpy as np


def _elsize(dtype) -> int:
    return np.dtype(dtype).itemsize


@dataclass(eq=False)
class ContractRequest:
    """C[indC] = alpha * A[indA] * B[indB] + beta * C0.

    A and B are host arrays in column-major order (Julia layout) or the key of
    a resident operand.  C0 (host, column-major) is required when beta != 0.
    """
    A: Any
    indA: tuple
    B: Any
    indB: tuple
    indC: tuple
    alpha: complex = 1.0
    beta: complex = 0.0
    C0: Optional[np.ndarray] = None
    dtype: Any = np.float64
    tag: Any = None
    # filled by the server
    arrival: float = 0.0
    admitted: float = 0.0
    done: float = 0.0
    result: Optional[np.ndarray] = None
    error: Optional[str] = None
    _release: Any = None
    _prep: Any = None      # the backend's staged buffers and plan, once prepared
    prepared: bool = False
    _reserved: int = 0     # device bytes charged to the budget in preparation
    _pstate: int = 0       # preparation: 0 queued, 1 taken (by the thread or the loop)

    def release_result(self) -> None:
        """Hand the result's pinned host buffer back to the server's pool
        (the result array must not be used afterwards)."""
        if self._release is not None:
            fn, buf = self._release
            self._release = None
            self.result = None
            fn(buf)

    def c_shape(self, shape_of) -> tuple:
        sa, sb = shape_of(self.A), shape_of(self.B)
        dims = {}
        for lab, n in zip(self.indA, sa):
            dims[lab] = n
        for lab, n in zip(self.indB, sb):
            dims[lab] = n
        return tuple(dims[l] for l in self.indC)

    def flops(self, shape_of) -> float:
        """Algorithmic work: 2*M*N*K real, 8*M*N*K complex."""
        sa, sb = shape_of(self.A), shape_of(self.B)
        size = {}
        for lab, n in list(zip(self.indA, sa)) + list(zip(self.indB, sb)):
            size[lab] = n
        mnk = 1  # every label is in exactly two operands: the product is M*N*K
        for n in size.values():
            mnk *= n
        return (8.0 if np.issubdtype(np.dtype(self.dtype), np.complexfloating) else 2.0) * mnk


@dataclass(eq=False)
class Tick:
    requests: list
    bytes: int
    handle: Any = None
    launched: float = 0.0


def percentile(xs: Sequence[float], q: float) -> float:
    """Nearest-rank percentile (q in [0, 100])."""
    if not xs:
        return float("nan")
    s = sorted(xs)
    k = max(1, int(math.ceil(q / 100.0 * len(s))))
    return s[k - 1]


class ContractionServer:
    """Continuous-batching server over a backend (``DeviceBackend`` on a GPU)."""

    def __init__(self, backend, hbm_budget_bytes: int = 120 << 30, max_ticks: int = 4,
                 max_tick_requests: int = 512, max_tick_bytes: Optional[int] = None,
                 max_tick_flops: Optional[float] = None, on_done=None):
        self.be = backend
        # A tick ends when it holds max_tick_flops of work (at least one
        # request): short ticks pipeline, and small requests are not held
        # back behind a long tick.
        self.max_tick_flops = max_tick_flops
        self.on_done = on_done  # called with each completed request
        self.budget = int(hbm_budget_bytes)
        self.max_ticks = int(max_ticks)
        self.max_tick_requests = int(max_tick_requests)
        self.max_tick_bytes = max_tick_bytes
        self.used = 0                      # bytes held by in-flight ticks + residents
        self.peak_used = 0
        self.pending = collections.deque()
        self.inflight: list[Tick] = []
        self.completed: list[ContractRequest] = []
        self.residents: dict = {}
        self._lock = threading.Lock()
        self._inbox = collections.deque()
        self.ticks_launched = 0
        # A backend with `prepare` (staging and planning per request) gets a
        # preparation thread: requests are prepared as they arrive, off the
        # loop that completes, admits and launches ticks.
        self._prepare = getattr(backend, "prepare", None)
        self._prep_q = collections.deque()
        self._prep_cv = threading.Condition()
        self._budget_cv = threading.Condition()  # guards `used` while preparation runs
        self._prep_stop = False
        self._prep_thread = None
        if self._prepare is not None:
            self._prep_thread = threading.Thread(target=self._prep_loop, name="qs-serve-prepare", daemon=True)
            self._prep_thread.start()

    def _prep_loop(self) -> None:
        while True:
            with self._prep_cv:
                while not self._prep_q and not self._prep_stop:
                    self._prep_cv.wait()
                if self._prep_stop:
                    return
                r = self._prep_q.popleft()
                if r._pstate != 0:  # the loop took it
                    continue
                r._pstate = 1
            self._prepare_now(r, wait=True)

    def _prepare_now(self, r: ContractRequest, wait: bool) -> bool:
        """Reserve and prepare r; False (r untouched, back in the queue's
        state) when wait is False and its bytes do not fit yet."""
        try:
            ok = self._reserve(r, wait)
            if ok is None:
                with self._prep_cv:
                    r._pstate = 0
                return False
            if ok:
                self._prepare(r)
        except Exception as e:  # the request fails alone; the loop reports it
            r.error = f"preparation failed: {e}"
        r.prepared = True
        return True

    def _reserve(self, r: ContractRequest, wait: bool = True):
        """Charge a request's device bytes to the budget before it is staged
        (waiting for completions while it does not fit, or returning None at
        once when wait is False); False for a request larger than the
        budget, which fails."""
        b = self.request_bytes(r)
        with self._budget_cv:
            if b > self.budget - sum(self.residents.values()):
                r.error = f"request needs {b} bytes, more than the budget"
                return False
            while self.used + b + self.be.cached_bytes() > self.budget:
                self.be.evict(self.used + b + self.be.cached_bytes() - self.budget)
                if self.used + b + self.be.cached_bytes() <= self.budget or self._prep_stop:
                    break
                if not wait:
                    return None
                self._budget_cv.wait(0.01)
            self.used += b
            self.peak_used = max(self.peak_used, self.used)
        r._reserved = b
        return True

    def close(self) -> None:
        """Stop the preparation thread (requests not yet prepared are
        prepared by the loop when admitted)."""
        if self._prep_thread is not None:
            with self._prep_cv:
                self._prep_stop = True
                self._prep_cv.notify()
            self._prep_thread.join()
            self._prep_thread = None
            self._prepare = None

    # ------------------------------------------------------------ API ---
    def put_resident(self, key, array) -> None:
        nbytes = self.be.put_resident(key, array)
        with self._budget_cv:
            self.residents[key] = nbytes
            self.used += nbytes
            self.peak_used = max(self.peak_used, self.used)

    def drop_resident(self, key) -> None:
        self.be.drop_resident(key)
        with self._budget_cv:
            self.used -= self.residents.pop(key)
            self._budget_cv.notify_all()

    def submit(self, req: ContractRequest, now: Optional[float] = None) -> ContractRequest:
        req.arrival = time.perf_counter() if now is None else now
        with self._lock:
            self._inbox.append(req)
        if self._prepare is not None:
            with self._prep_cv:
                self._prep_q.append(req)
                self._prep_cv.notify()
        return req

    def request_bytes(self, req: ContractRequest) -> int:
        return self.be.request_bytes(req)

    # ----------------------------------------------------------- loop ---
    def step(self) -> bool:
        """One tick of the loop; returns True when anything happened."""
        busy = False
        with self._lock:
            while self._inbox:
                self.pending.append(self._inbox.popleft())
        # 1. completions, in launch order
        still = []
        for t in self.inflight:
            if self.be.tick_done(t.handle):
                now = time.perf_counter()
                self.be.finish_tick(t.handle, t.requests)
                for r in t.requests:
                    r.done = now
                    self.completed.append(r)
                    if self.on_done is not None:
                        self.on_done(r)
                with self._budget_cv:
                    self.used -= t.bytes
                    self._budget_cv.notify_all()
                busy = True
            else:
                still.append(t)
        self.inflight = still
        # 2. admission (FIFO; a request that does not fit waits, later ones too)
        if self.pending and len(self.inflight) < self.max_ticks:
            batch, nbytes, work, reserved = [], 0, 0.0, 0  # reserved: bytes charged in preparation
            while self.pending and len(batch) < self.max_tick_requests:
                r = self.pending[0]
                if self._prepare is not None:
                    if not r.prepared:
                        # FIFO: wait for its preparation, or do it here when
                        # the preparation thread has not started it
                        with self._prep_cv:
                            mine = r._pstate == 0
                            if mine:
                                r._pstate = 1
                        if not (mine and self._prepare_now(r, wait=False)):
                            break
                    if r.error is not None:  # rejected or failed in preparation
                        self.pending.popleft()
                        with self._budget_cv:
                            self.used -= r._reserved
                            self._budget_cv.notify_all()
                        r._reserved = 0
                        r.done = time.perf_counter()
                        self.completed.append(r)
                        continue
                    f = r.flops(self.be.shape_of) if self.max_tick_flops else 0.0
                    if self.max_tick_flops and batch and work + f > self.max_tick_flops:
                        break
                    if self.max_tick_bytes and batch and nbytes + r._reserved > self.max_tick_bytes:
                        break
                    batch.append(self.pending.popleft())
                    reserved += r._reserved
                    nbytes += r._reserved
                    work += f
                    continue
                b = self.request_bytes(r)
                f = r.flops(self.be.shape_of) if self.max_tick_flops else 0.0
                if self.max_tick_flops and batch and work + f > self.max_tick_flops:
                    break
                if b > self.budget - sum(self.residents.values()):
                    self.pending.popleft()
                    r.error = f"request needs {b} bytes, more than the budget"
                    r.done = time.perf_counter()
                    self.completed.append(r)
                    continue
                if self.used + nbytes + b + self.be.cached_bytes() > self.budget:
                    # cached plan workspaces are the first to go
                    self.be.evict(self.used + nbytes + b + self.be.cached_bytes() - self.budget)
                    if self.used + nbytes + b + self.be.cached_bytes() > self.budget:
                        break
                if self.max_tick_bytes and batch and nbytes + b > self.max_tick_bytes:
                    break
                batch.append(self.pending.popleft())
                nbytes += b
                work += f
            if batch:
                now = time.perf_counter()
                for r in batch:
                    r.admitted = now
                with self._budget_cv:
                    self.used += nbytes - reserved
                    self.peak_used = max(self.peak_used, self.used)
                handle = self.be.launch_tick(batch)
                self.inflight.append(Tick(batch, nbytes, handle, now))
                self.ticks_launched += 1
                busy = True
        return busy

    def idle(self) -> bool:
        with self._lock:
            inbox = len(self._inbox)
        return not self.pending and not self.inflight and inbox == 0

    def drain(self, timeout: float = 600.0) -> None:
        t0 = time.perf_counter()
        while not self.idle():
            if not self.step():
                time.sleep(20e-6)
            if time.perf_counter() - t0 > timeout:
                raise TimeoutError("serving loop did not drain")

    def replay(self, requests: Sequence[ContractRequest], offsets: Sequence[float],
               timeout: float = 600.0) -> float:
        """Submit requests[i] at start + offsets[i] (seconds) while running the
        loop; returns the wall time from the first arrival to the last
        completion."""
        order = sorted(range(len(requests)), key=lambda i: offsets[i])
        start = time.perf_counter()
        k = 0
        while k < len(order) or not self.idle():
            now = time.perf_counter()
            while k < len(order) and start + offsets[order[k]] <= now:
                i = order[k]
                self.submit(requests[i], now=start + offsets[i])
                k += 1
            if not self.step():
                time.sleep(20e-6)
            if now - start > timeout:
                raise TimeoutError("replay did not finish")
        return time.perf_counter() - start

    def stats(self, requests: Optional[Sequence[ContractRequest]] = None) -> dict:
        reqs = list(requests) if requests is not None else self.completed
        lat = [1e3 * (r.done - r.arrival) for r in reqs if r.error is None]
        return {"requests": len(reqs), "errors": sum(1 for r in reqs if r.error),
                "p50_ms": percentile(lat, 50), "p99_ms": percentile(lat, 99),
                "mean_ms": float(np.mean(lat)) if lat else float("nan"),
                "ticks": self.ticks_launched, "peak_bytes": self.peak_used}


def serve_sequential(backend, requests: Sequence[ContractRequest], offsets: Sequence[float],
                     on_done=None) -> float:
    """Baseline: one request at a time in arrival order (upload, plan, one
    execute, download, wait), each starting no earlier than its arrival."""
    order = sorted(range(len(requests)), key=lambda i: offsets[i])
    start = time.perf_counter()
    for i in order:
        r = requests[i]
        t_arr = start + offsets[i]
        while time.perf_counter() < t_arr:
            time.sleep(20e-6)
        r.arrival = t_arr
        r.admitted = time.perf_counter()
        h = backend.launch_tick([r], grouped=False)
        while not backend.tick_done(h):
            time.sleep(10e-6)
        backend.finish_tick(h, [r])
        r.done = time.perf_counter()
        if on_done is not None:
            on_done(r)
    return time.perf_counter() - start


class Arena:
    """First-fit allocator over one preallocated byte range (offsets only).
    Blocks are aligned to `align` bytes; freed neighbours merge."""

    def __init__(self, capacity: int, align: int = 256):
        self.capacity = int(capacity)
        self.align = align
        self.free_list = [(0, self.capacity)] if capacity > 0 else []  # sorted (offset, size)
        self.live = {}

    def alloc(self, nbytes: int) -> Optional[int]:
        n = max(self.align, (int(nbytes) + self.align - 1) // self.align * self.align)
        for i, (off, size) in enumerate(self.free_list):
            if size >= n:
                if size == n:
                    self.free_list.pop(i)
                else:
                    self.free_list[i] = (off + n, size - n)
                self.live[off] = n
                return off
        return None

    def free(self, off: int) -> None:
        n = self.live.pop(off)
        fl = self.free_list
        lo, hi = 0, len(fl)
        while lo < hi:
            mid = (lo + hi) // 2
            if fl[mid][0] < off:
                lo = mid + 1
            else:
                hi = mid
        fl.insert(lo, (off, n))
        # merge with the right, then the left neighbour
        if lo + 1 < len(fl) and fl[lo][0] + fl[lo][1] == fl[lo + 1][0]:
            fl[lo] = (fl[lo][0], fl[lo][1] + fl[lo + 1][1])
            fl.pop(lo + 1)
        if lo > 0 and fl[lo - 1][0] + fl[lo - 1][1] == fl[lo][0]:
            fl[lo - 1] = (fl[lo - 1][0], fl[lo - 1][1] + fl[lo][1])
            fl.pop(lo)

    def used(self) -> int:
        return sum(self.live.values())


# ------------------------------------------------------------ device ---

class DeviceBackend:
    """The engine on one GPU: torch for device memory, streams and events;
    plans and grouped launches through the C ABI."""

    def __init__(self, qs, device: int = 0, nstreams: int = 4, grouped: bool = True,
                 device_arena_bytes: int = 1 << 30, host_arena_bytes: int = 256 << 20):
        import torch
        self.torch = torch
        self.qs = qs
        self.dev = torch.device("cuda", device)
        # Request buffers come from two arenas allocated once: device memory
        # for operands and C, pinned host memory for results and staging.
        # Allocating either per request costs milliseconds per GB and can
        # wait on work in flight.
        self.dev_mem = torch.empty(int(device_arena_bytes), dtype=torch.uint8, device=self.dev)
        self.host_mem = torch.empty(int(host_arena_bytes), dtype=torch.uint8, pin_memory=True)
        self.dev_arena = Arena(device_arena_bytes)
        self.host_arena = Arena(host_arena_bytes)
        self.fallbacks = collections.Counter()
        self.streams = [torch.cuda.Stream(device=self.dev) for _ in range(nstreams)]
        self.next_stream = 0
        self.resident = {}
        self.plan_cache = collections.OrderedDict()  # signature -> [plans], LRU first
        self._cached_bytes = 0
        self.grouped = grouped
        # The server's preparation thread and its loop share the arenas and
        # the plan cache (_lock) and call into the library (_qs_lock: one
        # library call at a time; a plan or a grouped launch takes tens of
        # microseconds).
        self._lock = threading.RLock()
        self._qs_lock = threading.RLock()
        # host seconds per launch phase, and device milliseconds per tick
        self.timing = collections.Counter()
        self.tick_gpu_ms = []
        self._tdtype = {np.dtype(np.float32): torch.float32, np.dtype(np.float64): torch.float64,
                        np.dtype(np.complex64): torch.complex64, np.dtype(np.complex128): torch.complex128}

    def _take(self, arena, mem, n, tdt, where):
        """(handle, tensor of n elements): a block of the arena, or a fresh
        allocation when the arena is full (counted in `fallbacks`)."""
        es = self.torch.empty((), dtype=tdt).element_size()
        off = arena.alloc(n * es)
        if off is None:
            self.fallbacks[where] += 1
            t = (self.torch.empty(n, dtype=tdt, pin_memory=True) if where == "host"
                 else self.torch.empty(n, dtype=tdt, device=self.dev))
            return (None, None), t
        return (arena, off), mem[off:off + n * es].view(tdt)

    def _pinned(self, n, tdt):
        return self._take(self.host_arena, self.host_mem, n, tdt, "host")

    def _device(self, n, tdt):
        return self._take(self.dev_arena, self.dev_mem, n, tdt, "device")

    def _give(self, handle):
        arena, off = handle
        if arena is not None:
            with self._lock:
                arena.free(off)

    def _unpin(self, handle):
        self._give(handle)

    # shapes of host arrays or resident keys
    def shape_of(self, x):
        if isinstance(x, str) or not hasattr(x, "shape"):
            return tuple(self.resident[x][1])
        return tuple(x.shape)

    def put_resident(self, key, array) -> int:
        arr = np.asfortranarray(array)
        t = self.torch.from_numpy(arr.ravel(order="F").copy()).to(self.dev)
        self.resident[key] = (t, arr.shape, arr.dtype)
        return t.numel() * t.element_size()

    def drop_resident(self, key) -> None:
        del self.resident[key]

    def request_bytes(self, r: ContractRequest) -> int:
        es = _elsize(r.dtype)
        n = 0
        for x in (r.A, r.B):
            if not isinstance(x, str):
                n += int(np.prod(x.shape)) * es
        nc = int(np.prod(r.c_shape(self.shape_of))) if r.indC else 1
        n += nc * es
        # tensor-core workspace: at most ~1 byte per operand element per slice
        return n + (n * 7) // 8

    @staticmethod
    def _colmajor(shape):
        st, acc = [], 1
        for s in shape:
            st.append(acc)
            acc *= s
        return tuple(st)

    def _view(self, t, shape):
        return self.qs.StridedView(t, tuple(shape), self._colmajor(shape), 0)

    def _signature(self, r, sa, sb, sc):
        return (np.dtype(r.dtype).str, sa, tuple(r.indA), sb, tuple(r.indB), sc, tuple(r.indC))

    def prepare(self, r: ContractRequest) -> None:
        """Stage one request for its tick: device blocks for A, B and C,
        pinned copies of host operands, and its plan (from the plan cache
        or `plan_contract`).  The server runs this on its preparation
        thread as requests arrive, so the loop that admits and launches
        ticks does none of it; `launch_tick` only enqueues device work."""
        # The preparation thread's current device is not the loop's: plans
        # and their workspace go to this backend's device.
        with self.torch.cuda.device(self.dev):
            self._prepare_on_device(r)

    def _prepare_on_device(self, r: ContractRequest) -> None:
        torch = self.torch
        clk = time.perf_counter
        t0 = clk()
        tdt = self._tdtype[np.dtype(r.dtype)]
        staged, dev_blocks, copies_in = [], [], []

        def device_copy_of(x):
            h = torch.from_numpy(np.asfortranarray(x).ravel(order="F"))
            if not h.is_pinned():
                with self._lock:
                    buf, h2 = self._pinned(h.numel(), tdt)
                h2.copy_(h)
                staged.append(buf)
                h = h2
            with self._lock:
                dh, t = self._device(h.numel(), tdt)
            dev_blocks.append(dh)
            copies_in.append((t, h))
            return t

        ops = []
        for x in (r.A, r.B):
            if isinstance(x, str):
                t, shp, _ = self.resident[x]
                ops.append((t, shp))
            else:
                ops.append((device_copy_of(x), x.shape))
        sc = r.c_shape(self.shape_of)
        ncs = int(np.prod(sc)) if sc else 1
        zero_c = r.C0 is None
        if zero_c:
            with self._lock:
                dh, Cd = self._device(ncs, tdt)
            dev_blocks.append(dh)
        else:
            Cd = device_copy_of(r.C0)
        t1 = clk()
        Av, Bv, Cv = self._view(ops[0][0], ops[0][1]), self._view(ops[1][0], ops[1][1]), self._view(Cd, sc)
        key = self._signature(r, tuple(ops[0][1]), tuple(ops[1][1]), tuple(sc))
        plan = None
        with self._lock:
            if self.plan_cache.get(key):
                plan = self.plan_cache[key].pop()
                self._cached_bytes -= plan.workspace_bytes
        with self._qs_lock:
            if plan is not None:
                plan.rebind(Av, Bv, Cv)
            else:
                plan = self.qs.plan_contract(Cv, Av, r.indA, Bv, r.indB, r.indC)
        with self._lock:
            out_buf, host_out = self._pinned(ncs, tdt)
            self.timing["stage"] += t1 - t0
            self.timing["plan"] += clk() - t1
        r._prep = {"item": (r, key, plan, Cd, host_out, ops, sc, out_buf, staged, dev_blocks),
                   "copies_in": copies_in, "alpha": r.alpha, "beta": r.beta if not zero_c else 0.0}

    def launch_tick(self, batch, grouped: Optional[bool] = None):
        """Enqueue a tick's device work as one burst on the tick's stream:
        uploads, one grouped execute (or one execute per plan), downloads,
        an event.  Requests not yet prepared are prepared here."""
        torch = self.torch
        grouped = self.grouped if grouped is None else grouped
        st = self.streams[self.next_stream % len(self.streams)]
        self.next_stream += 1
        T = self.timing
        clk = time.perf_counter
        for r in batch:
            if getattr(r, "_prep", None) is None:
                self.prepare(r)
        items = [r._prep["item"] for r in batch]
        plans = [it[2] for it in items]
        alphas = [r._prep["alpha"] for r in batch]
        betas = [r._prep["beta"] for r in batch]
        with torch.cuda.stream(st):
            ev0 = torch.cuda.Event(enable_timing=True)
            ev0.record(st)
            for r in batch:
                for t, h in r._prep["copies_in"]:
                    t.copy_(h, non_blocking=True)
            t3 = clk()
            with self._qs_lock:
                if grouped and len(plans) > 1:  # one plan: its own execute, no group tables
                    g = self.qs.ContractGroup(plans, mode="persistent")
                    g.execute(alphas, betas, stream=st)
                else:
                    g = None
                    for p, a, b in zip(plans, alphas, betas):
                        self.qs.execute(p, a, b, stream=st)
            T["execute"] += clk() - t3
            for it in items:
                it[4].copy_(it[3], non_blocking=True)
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(st)
        for r in batch:
            r._prep = None
        T["ticks"] += 1
        return {"event": ev, "start": ev0, "items": items, "group": g, "stream": st}

    def tick_done(self, h) -> bool:
        return h["event"].query()

    def finish_tick(self, h, batch) -> None:
        h["event"].synchronize()
        self.tick_gpu_ms.append(h["start"].elapsed_time(h["event"]))
        if h["group"] is not None:
            with self._qs_lock:
                h["group"].release()
        # Each result is a view of a pooled pinned buffer, handed to the
        # request; ContractRequest.release_result() returns the buffer.
        for (r, key, plan, Cd, host_out, ops, sc, out_buf, staged, dev_blocks) in h["items"]:
            res = host_out.numpy()
            r.result = res.reshape(sc, order="F") if sc else res
            r._release = (self._unpin, out_buf)
            for b in staged:
                self._unpin(b)
            for b in dev_blocks:  # the tick's event has fired: the device is done with them
                self._give(b)
            with self._qs_lock:
                plan.detach_storage()
            with self._lock:
                self.plan_cache.setdefault(key, []).append(plan)
                self.plan_cache.move_to_end(key)
                self._cached_bytes += plan.workspace_bytes
        h["items"] = []

    def clear_plan_cache(self) -> None:
        """Release every cached plan."""
        with self._lock, self._qs_lock:
            for plans in self.plan_cache.values():
                for p in plans:
                    p.release()
            self.plan_cache.clear()
            self._cached_bytes = 0

    def cached_bytes(self) -> int:
        """Device workspace held by idle cached plans."""
        return self._cached_bytes

    def evict(self, nbytes: int) -> None:
        """Release least recently used cached plans until nbytes are freed."""
        freed = 0
        with self._lock, self._qs_lock:
            while freed < nbytes and self.plan_cache:
                key, plans = next(iter(self.plan_cache.items()))
                while plans and freed < nbytes:
                    p = plans.pop()
                    freed += p.workspace_bytes
                    self._cached_bytes -= p.workspace_bytes
                    p.release()
                if not plans:
                    del self.plan_cache[key]
