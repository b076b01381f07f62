"""Host-side mirror of QuasiStrided.jl's engine API over the B200 C-ABI library.

Names, argument meaning and error behaviour follow the reference:

====================  ==========================================================
this module           QuasiStrided.jl
====================  ==========================================================
``StridedView``       ``StridedViews.StridedView`` (parent, size, strides, offset, op)
``plan_contract``     ``plan_contract`` (src/planning/plan.jl:115-133)
``execute``           ``execute!`` (src/execution/execute.jl:11-20)
``contract``          ``contract!`` (src/execution/execute.jl:84-95)
``ContractPlan``      ``ContractPlan`` (src/planning/plan.jl:16-45)
``release``           ``release!`` (src/execution/workspace.jl:118-123)
``PathModes``         ``PathModes`` (src/planning/plan.jl:60-64)
``QuasiStridedBackend``  ``QuasiStridedBackend`` (src/integrations/tensoroperations.jl:24-32)
``tensorcontract``    ``TO.tensorcontract!`` method (tensoroperations.jl:75-88)
``contraction_labels``  ``contraction_labels`` (tensoroperations.jl:40-47)
====================  ==========================================================

Operands are ``StridedView`` s over torch tensors in device memory.  All
compute happens in libqsgpu.so's sm_100a kernels; there is no CPU fallback:
a missing library or a non-CUDA operand raises.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional, Sequence

import torch

from . import _abi
from .allocators import (DeviceArena, TorchAllocator, allocator_checkpoint,  # noqa: F401
                         allocator_handle, allocator_reset, tensoralloc, tensorfree)
from ._abi import (ArgumentError, BoundsError, DeviceTimeout, DimensionMismatch,  # noqa: F401
                   EngineError, QS_C32, QS_C64, QS_F32, QS_F64)

__all__ = [
    "StridedView", "plan_contract", "execute", "contract", "ContractPlan", "PathModes",
    "QuasiStridedBackend", "tensorcontract", "contraction_labels", "release",
    "ArgumentError", "DimensionMismatch", "BoundsError", "EngineError", "DeviceTimeout", "colmajor",
    "execute_grouped", "ContractGroup", "add_trace", "tensoradd", "tensortrace",
    "DeviceArena", "TorchAllocator", "tensoralloc", "tensorfree", "allocator_checkpoint",
    "allocator_reset", "check_status", "set_wait_limit",
]

_DTYPE_TO_QS = {torch.float32: QS_F32, torch.float64: QS_F64,
                torch.complex64: QS_C32, torch.complex128: QS_C64}
_OPS = ("identity", "conj", "transpose", "adjoint")


def _layout_of(v) -> tuple:
    return (tuple(v.size), tuple(v.strides), int(v.offset), int(v.parent.numel()), v.dtype, v.op)


def _eltype(dtype: torch.dtype) -> int:
    try:
        return _DTYPE_TO_QS[dtype]
    except KeyError:
        raise ArgumentError(
            f"plan_contract: eltype {dtype}; each must be one of Float32, Float64, "
            "ComplexF32, ComplexF64") from None


class StridedView:
    """A strided window (size, strides, offset, op) into a flat parent tensor.

    ``StridedView(t)`` wraps a torch tensor with its own size/strides/offset;
    ``StridedView(parent, size, strides, offset, op)`` builds one explicitly
    (StridedViews.jl's five-argument constructor).  Strides are in elements
    and may be zero or negative; nothing checks the window against the
    parent here — ``execute`` does, before any write.
    """

    def __init__(self, parent: torch.Tensor, size: Optional[Sequence[int]] = None,
                 strides: Optional[Sequence[int]] = None, offset: Optional[int] = None,
                 op: str = "identity"):
        if not isinstance(parent, torch.Tensor):
            raise ArgumentError("StridedView parent must be a torch.Tensor")
        if op not in _OPS:
            raise ArgumentError(
                f"unsupported StridedView.op {op}: QuasiStrided folds a view's `op` into the "
                "packing transform and recognizes only identity/conj/transpose/adjoint")
        if size is None:
            size, strides = tuple(parent.shape), tuple(parent.stride())
            offset = parent.storage_offset() if offset is None else offset
            n = parent.untyped_storage().nbytes() // parent.element_size()
            flat = torch.as_strided(parent, (n,), (1,), 0)
        else:
            if strides is None:
                raise ArgumentError("StridedView: strides are required with size")
            flat = parent.reshape(-1) if parent.dim() != 1 else parent
            offset = 0 if offset is None else offset
        self.parent = flat
        self.size = tuple(int(s) for s in size)
        self.strides = tuple(int(s) for s in strides)
        if len(self.size) != len(self.strides):
            raise ArgumentError("StridedView: size and strides differ in length")
        self.offset = int(offset)
        self.op = op

    @property
    def dtype(self):
        return self.parent.dtype

    @property
    def ndim(self):
        return len(self.size)

    def permutedims(self, perm: Sequence[int]) -> "StridedView":
        """permutedims(view, perm), 0-based perm."""
        return StridedView(self.parent, [self.size[p] for p in perm],
                           [self.strides[p] for p in perm], self.offset, self.op)

    def with_op(self, op: str) -> "StridedView":
        return StridedView(self.parent, self.size, self.strides, self.offset, op)

    def to_tensor(self) -> torch.Tensor:
        """Materialise the window (applying a conjugating op), for tests."""
        t = torch.as_strided(self.parent, self.size, self.strides, self.offset) if self.size else \
            self.parent[self.offset:self.offset + 1].reshape(())
        if self.op in ("conj", "adjoint") and t.is_complex():
            t = t.conj()
        return t.resolve_conj()

    def _c(self, keep: list) -> _abi.qs_view:
        size = (ctypes.c_int64 * max(1, len(self.size)))(*self.size)
        strides = (ctypes.c_int64 * max(1, len(self.strides)))(*self.strides)
        keep.extend([size, strides])
        v = _abi.qs_view()
        v.data = self.parent.data_ptr()
        v.length = self.parent.numel()
        v.offset = self.offset
        v.size = size
        v.strides = strides
        v.ndim = len(self.size)
        v.eltype = _eltype(self.parent.dtype)
        v.op = _abi.QS_OP[self.op]
        return v


def colmajor(shape: Sequence[int], dtype=torch.float64, device="cuda", fill=None,
             generator=None) -> StridedView:
    """A dense column-major (Julia layout) array as a StridedView."""
    n = 1
    for s in shape:
        n *= int(s)
    if fill is None:
        parent = torch.zeros(max(n, 1), dtype=dtype, device=device)
    else:
        parent = torch.full((max(n, 1),), fill, dtype=dtype, device=device)
    strides, acc = [], 1
    for s in shape:
        strides.append(acc)
        acc *= int(s)
    return StridedView(parent, tuple(shape), tuple(strides), 0)


@dataclass(frozen=True)
class PathModes:
    """Overrides for the dot / outer-product / read-B-in-place paths
    (``:auto``/``:never``/``:always`` in the reference)."""
    dot: str = "auto"
    outer: str = "auto"
    unpacked_b: str = "auto"


def _acc_code(accumulator) -> int:
    if accumulator in (None, "nothing"):
        return 0
    if accumulator in ("Float32", torch.float32):
        return 1
    if accumulator in ("Float64", torch.float64):
        return 2
    raise ArgumentError(
        f"QuasiStridedBackend: accumulator must be nothing, Float32 or Float64, got {accumulator}")


def _scalar(x) -> ctypes.Array:
    if isinstance(x, torch.Tensor):
        x = x.item()
    z = complex(x)
    return (ctypes.c_double * 2)(z.real, z.imag)


class ContractPlan:
    """Reusable plan: M/N/K groups, path, method and the device workspace.

    The plan borrows the operands' storage (it keeps the Python objects
    alive) and owns its workspace until ``release``.  One execution at a time.
    """

    def __init__(self, handle, C, A, B, host_only):
        self._h = handle
        self.C, self.A, self.B = C, A, B
        self._layout = {"A": _layout_of(A), "B": _layout_of(B), "C": _layout_of(C)}
        self.host_only = host_only
        info = _abi.qs_plan_info()
        _abi.check(_abi.lib().qs_plan_get_info(handle, ctypes.byref(info)))
        self.path = _abi.QS_PATH_NAME[info.path]
        self.method = _abi.QS_METHOD_NAME[info.method]
        self.compute_type = _abi.ELTYPE_NAME[info.compute_type]
        self.swapped = bool(info.swapped)
        self.conjA, self.conjB = bool(info.conjA), bool(info.conjB)
        self.ozaki_slices = info.ozaki_slices
        self.complex_mode = {0: None, 1: "planar", 2: "1m"}[info.complex_mode]
        self.m_length, self.n_length, self.k_length = info.m_length, info.n_length, info.k_length
        self.m_labels = tuple(info.m_labels[:info.m_rank])
        self.n_labels = tuple(info.n_labels[:info.n_rank])
        self.k_labels = tuple(info.k_labels[:info.k_rank])
        self.bounds_ok = bool(info.bounds_ok)
        self.workspace_bytes = info.workspace_bytes
        self.stride_class = info.stride_class
        self.native_tile = info.native_tile
        self.oz_single_sm = False
        self.batch_labels = tuple(info.batch_labels[:info.batch_rank])
        self.batch_length = info.batch_length

    @property
    def Cstorage(self) -> torch.Tensor:
        return self.C.parent

    def rebind(self, A: Optional[StridedView] = None, B: Optional[StridedView] = None,
               C: Optional[StridedView] = None) -> None:
        """Point the plan at new storage with the same layout (size, strides,
        offset, parent length, eltype and op as at plan time); qs_plan_rebind."""
        def same(new, name):
            if new is None:
                if getattr(self, name) is None:
                    raise ArgumentError(f"rebind: {name} has no storage bound")
                return None
            if _layout_of(new) != self._layout[name]:
                raise ArgumentError(f"rebind: {name} differs in layout from the planned view")
            return ctypes.c_void_p(new.parent.data_ptr())
        pa, pb, pc = same(A, "A"), same(B, "B"), same(C, "C")
        _abi.check(_abi.lib().qs_plan_rebind(self._h, pa, pb, pc))
        self.A = A if A is not None else self.A
        self.B = B if B is not None else self.B
        self.C = C if C is not None else self.C

    def detach_storage(self) -> None:
        """Drop the plan's references to its operands (their memory may then
        be freed); the plan executes again only after ``rebind``."""
        self.A = self.B = self.C = None

    def release(self) -> None:
        if self._h:
            _abi.lib().qs_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    def __repr__(self):
        return (f"ContractPlan({self.compute_type}, {self.path}, method={self.method}, "
                f"M={self.m_length}, N={self.n_length}, K={self.k_length}, swapped={self.swapped})")


def _options(conjA=False, conjB=False, accumulator=None, method="auto", m_block=None,
             k_block=None, n_block=None, path_modes: Optional[PathModes] = None,
             ozaki_slices=0, complex_mode=None, host_only=False,
             per_product_gemm=False, cuda_graph=False, batch_labels=False,
             oz_single_sm=False) -> _abi.qs_plan_options:
    o = _abi.qs_plan_options()
    o.conjA, o.conjB = int(bool(conjA)), int(bool(conjB))
    o.accumulator = _acc_code(accumulator)
    if method not in _abi.QS_METHOD:
        raise ArgumentError(f"unknown method {method!r}")
    o.method = _abi.QS_METHOD[method]
    for name, val in (("m_block", m_block), ("k_block", k_block), ("n_block", n_block)):
        if val is not None and int(val) < 1:
            raise ArgumentError(f"{name} must be >= 1, got {val}")
        setattr(o, name, 0 if val is None else int(val))
    pm = path_modes or PathModes()
    o.dot_mode = _abi.QS_MODE[pm.dot]
    o.outer_mode = _abi.QS_MODE[pm.outer]
    o.unpacked_b_mode = _abi.QS_MODE[pm.unpacked_b]
    o.ozaki_slices = int(ozaki_slices)
    o.complex_mode = _abi.QS_CPLX[complex_mode]
    o.flags = ((_abi.QS_PLAN_HOST_ONLY if host_only else 0) | (2 if per_product_gemm else 0) |
               (4 if cuda_graph else 0) | (_abi.QS_PLAN_BATCH_LABELS if batch_labels else 0) |
               (_abi.QS_PLAN_OZ_SINGLE_SM if oz_single_sm else 0))
    return o


def _labels(ind: Sequence[int], n: int, name: str, keep: list):
    ind = tuple(int(x) for x in ind)
    if len(ind) != n:
        raise ArgumentError(f"{name} has {len(ind)} labels for a rank-{n} operand")
    arr = (ctypes.c_int64 * max(1, n))(*ind)
    keep.append(arr)
    return arr


def _check_device(host_only: bool, *views: StridedView) -> None:
    if host_only:
        return
    for v in views:
        if not v.parent.is_cuda:
            raise ArgumentError("operands must live in CUDA device memory (no CPU fallback)")


def plan_contract(C: StridedView, A: StridedView, indA, B: StridedView, indB, indC, *,
                  kernel=None, conjA=False, conjB=False, m_block=None, k_block=None,
                  n_block=None, allocator=None, accumulator=None,
                  path_modes: Optional[PathModes] = None, method="auto", ozaki_slices=0,
                  complex_mode=None, host_only=False, per_product_gemm=False,
                  cuda_graph=False, native_tile=0, batch_labels=False,
                  oz_single_sm=False) -> ContractPlan:
    """Plan ``C[indC] = A[indA] * B[indB]`` (every label in exactly two operands).

    Throws ArgumentError / DimensionMismatch on invalid input, before any
    device work.  ``kernel`` names a method ("native", "ozaki", "bf16x3");
    ``cuda_graph`` makes ``execute`` replay a captured CUDA graph of the
    plan's launches (re-captured when alpha/beta change);
    ``oz_single_sm=True`` runs the Ozaki GEMM (6 or 7 slices) on the one-SM
    kernel instead of the CTA-pair kernel.  ``batch_labels=True`` accepts labels present in A, B and C (the
    reference rejects them) as batch labels: one contraction per batch entry.
    ``allocator`` serves the plan's device workspace (None: the library's
    pool; a ``DeviceArena`` or ``TorchAllocator``), handed back in reverse
    order by ``release``; it must outlive the plan.  ``host_only`` plans
    without touching the device (inspection only).
    """
    if kernel is not None:
        method = kernel
    _check_device(host_only, C, A, B)
    keep: list = []
    cC, cA, cB = C._c(keep), A._c(keep), B._c(keep)
    iA = _labels(indA, A.ndim, "indA", keep)
    iB = _labels(indB, B.ndim, "indB", keep)
    iC = _labels(indC, C.ndim, "indC", keep)
    o = _options(conjA, conjB, accumulator, method, m_block, k_block, n_block, path_modes,
                 ozaki_slices, complex_mode, host_only, per_product_gemm, cuda_graph, batch_labels,
                 oz_single_sm)
    o.native_tile = int(native_tile)
    o.allocator = None if host_only else allocator_handle(allocator)
    h = ctypes.c_void_p()
    _abi.check(_abi.lib().qs_plan_contract(ctypes.byref(h), ctypes.byref(cC), ctypes.byref(cA), iA,
                                           ctypes.byref(cB), iB, iC, ctypes.byref(o)))
    plan = ContractPlan(h, C, A, B, host_only)
    plan.per_product_gemm, plan.cuda_graph = bool(per_product_gemm), bool(cuda_graph)
    plan.oz_single_sm = bool(oz_single_sm)
    plan.allocator = allocator
    return plan


def _stream_ptr(stream) -> Optional[int]:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


def execute(plan: ContractPlan, alpha, beta, stream=None) -> torch.Tensor:
    """``execute!``: C = alpha*A*B + beta*C for the plan; returns C's storage.

    beta applies exactly once and beta == 0 never reads C; alpha == 0 or an
    empty K never reads A or B; an out-of-bounds operand raises BoundsError
    before any write.  Enqueued on ``stream`` (default: torch's current).
    """
    if plan._h is None:
        raise ArgumentError("plan has been released")
    if plan.C is None or plan.A is None or plan.B is None:
        raise ArgumentError("plan has no storage bound (detached): rebind it first")
    a, b = _scalar(alpha), _scalar(beta)
    s = None if plan.host_only else _stream_ptr(stream)
    _abi.check(_abi.lib().qs_execute(plan._h, a, b, s))
    return plan.Cstorage


def profile(plan: ContractPlan, enable: bool = True) -> None:
    """Record CUDA events between the plan's launches on each execute."""
    _abi.check(_abi.lib().qs_plan_profile(plan._h, int(bool(enable))))


def stage_times(plan: ContractPlan):
    """Summed milliseconds per launch stage since profiling was enabled, and
    the number of executes recorded (synchronizes on the events)."""
    ms = (ctypes.c_double * 8)()
    ns, nx = ctypes.c_int32(), ctypes.c_int32()
    _abi.check(_abi.lib().qs_plan_stage_times(plan._h, ms, 8, ctypes.byref(ns), ctypes.byref(nx)))
    return [ms[i] for i in range(ns.value)], nx.value


def check_status(plan: ContractPlan, stream=None) -> None:
    """Raise EngineError if a tensor-core kernel of this plan gave up a
    bounded wait since the last check (synchronizes the stream)."""
    _abi.check(_abi.lib().qs_plan_check_status(plan._h, _stream_ptr(stream)))


def set_wait_limit(plan: ContractPlan, limit_ns: int = 0, hold_loads: bool = False) -> None:
    """Bound every device wait of the plan's tensor-core kernels by `limit_ns`
    (0: the default 2 s).  `hold_loads` is for failure-detection tests: the
    GEMM's producers issue no copies, so the first wait for operand tiles
    runs out and the kernel stops with QS_ETIMEOUT (nothing in flight, C
    untouched).  qs_plan_set_wait_limit."""
    _abi.check(_abi.lib().qs_plan_set_wait_limit(plan._h, int(limit_ns), int(bool(hold_loads))))


def release(plan: ContractPlan, allocator=None) -> None:
    """``release!``: free the plan's device workspace."""
    plan.release()


def contract(C: StridedView, alpha, A: StridedView, indA, B: StridedView, indB, beta, indC, *,
             accumulator=None, conjA=False, conjB=False, method="auto", stream=None,
             allocator=None, batch_labels=False) -> StridedView:
    """``contract!``: plan, execute, release; returns C.  With the library's
    pool this waits for the stream; with an ``allocator`` it returns once the
    work is enqueued (a ``DeviceArena`` is bracketed by checkpoint/reset, as
    TO.tensorcontract! brackets its allocator)."""
    _check_device(False, C, A, B)
    keep: list = []
    cC, cA, cB = C._c(keep), A._c(keep), B._c(keep)
    iA = _labels(indA, A.ndim, "indA", keep)
    iB = _labels(indB, B.ndim, "indB", keep)
    iC = _labels(indC, C.ndim, "indC", keep)
    o = _options(conjA, conjB, accumulator, method, batch_labels=batch_labels)
    o.allocator = allocator_handle(allocator)
    cp = allocator_checkpoint(allocator)
    try:
        _abi.check(_abi.lib().qs_contract(ctypes.byref(cC), _scalar(alpha), ctypes.byref(cA), iA,
                                          ctypes.byref(cB), iB, _scalar(beta), iC, ctypes.byref(o),
                                          _stream_ptr(stream)))
    finally:
        if cp is not None:
            allocator_reset(allocator, cp, stream)
    return C


def _scalar_pairs(values, n):
    arr = (ctypes.c_double * (2 * max(1, n)))()
    for i in range(n):
        z = complex(values[i])
        arr[2 * i], arr[2 * i + 1] = z.real, z.imag
    return arr


class ContractGroup:
    """Many independent plans executed together (qs_group_*).

    mode: "persistent" (one launch per stage and kernel class, over a device
    problem table), "sequential" (one execute per plan) — either with
    graph=True to capture the launches into a CUDA graph replayed on later
    executes.  The plans stay owned by the caller and must outlive the group.
    """

    def __init__(self, plans: Sequence[ContractPlan], mode: str = "persistent", graph: bool = False):
        modes = {"persistent": _abi.QS_GROUP_PERSISTENT, "sequential": _abi.QS_GROUP_SEQUENTIAL}
        if mode not in modes:
            raise ArgumentError(f"unknown group mode {mode!r}")
        self.plans = list(plans)
        n = len(self.plans)
        arr = (ctypes.c_void_p * max(1, n))(*[p._h for p in self.plans])
        h = ctypes.c_void_p()
        flag = modes[mode] | (_abi.QS_GROUP_GRAPH if graph else 0)
        _abi.check(_abi.lib().qs_group_create(n, arr, flag, ctypes.byref(h)))
        self._h = h
        self.mode, self.graph = mode, graph

    def execute(self, alphas, betas, stream=None) -> None:
        n = len(self.plans)
        if len(alphas) != n or len(betas) != n:
            raise ArgumentError("one alpha and one beta per plan")
        _abi.check(_abi.lib().qs_group_execute(self._h, _scalar_pairs(alphas, n), _scalar_pairs(betas, n),
                                               _stream_ptr(stream)))

    def info(self) -> dict:
        inf = _abi.qs_group_info()
        _abi.check(_abi.lib().qs_group_get_info(self._h, ctypes.byref(inf)))
        return {k: getattr(inf, k) for k, _ in _abi.qs_group_info._fields_}

    def release(self) -> None:
        if getattr(self, "_h", None):
            _abi.lib().qs_group_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


def execute_grouped(plans: Sequence[ContractPlan], alphas, betas, stream=None) -> None:
    """One-shot grouped execute (persistent mode); waits for the stream."""
    n = len(plans)
    arr = (ctypes.c_void_p * max(1, n))(*[p._h for p in plans])
    _abi.check(_abi.lib().qs_execute_grouped(n, arr, _scalar_pairs(alphas, n), _scalar_pairs(betas, n),
                                             _stream_ptr(stream)))


# ------------------------------------------------------- TensorOperations ---

def contraction_labels(pA, pB, pAB):
    """TO's (pA, pB, pAB) index tuples (1-based) -> (indA, indB, indC)."""
    NoA, Nk = len(pA[0]), len(pA[1])
    NoB = len(pB[1])
    if len(pB[0]) != Nk:
        raise ArgumentError("pA and pB disagree on the number of contracted indices")
    lin = lambda p: tuple(p[0]) + tuple(p[1])  # noqa: E731
    a, b, c = lin(pA), lin(pB), lin(pAB)
    mk = lambda xs: (ctypes.c_int64 * max(1, len(xs)))(*xs)  # noqa: E731
    outA = (ctypes.c_int64 * max(1, NoA + Nk))()
    outB = (ctypes.c_int64 * max(1, Nk + NoB))()
    outC = (ctypes.c_int64 * max(1, NoA + NoB))()
    _abi.check(_abi.lib().qs_contraction_labels(NoA, Nk, NoB, mk(a), mk(b), mk(c), outA, outB, outC))
    return tuple(outA[:NoA + Nk]), tuple(outB[:Nk + NoB]), tuple(outC[:NoA + NoB])


class QuasiStridedBackend:
    """TensorOperations-style backend running contractions on this engine.

    ``accumulator`` is ``None``, ``"Float32"`` or ``"Float64"`` and is
    validated at construction, as ``QuasiStridedBackend{A}()`` does.
    """

    def __init__(self, accumulator=None):
        _acc_code(accumulator)
        self.accumulator = accumulator

    def __repr__(self):
        return f"QuasiStridedBackend(accumulator={self.accumulator})"


def add_trace(C: StridedView, alpha, A: StridedView, indA, beta, indC, *, conjA=False, stream=None):
    """C[indC] = alpha * sum over the traced labels of op(A)[indA] + beta * C
    on the device (qs_tensoradd_trace): labels of indC appear once in indA,
    the other labels of indA exactly twice (traced pairs)."""
    _check_device(False, C, A, A)
    keep: list = []
    cC, cA = C._c(keep), A._c(keep)
    iA = _labels(indA, A.ndim, "indA", keep)
    iC = _labels(indC, C.ndim, "indC", keep)
    _abi.check(_abi.lib().qs_tensoradd_trace(ctypes.byref(cC), _scalar(alpha), ctypes.byref(cA), iA,
                                             int(bool(conjA)), _scalar(beta), iC, _stream_ptr(stream)))
    return C


def _as_view(x):
    return x if isinstance(x, StridedView) else StridedView(x)


def tensoradd(C, A, pA, conjA, alpha, beta, backend: "QuasiStridedBackend" = None, allocator=None):
    """``TO.tensoradd!(C, A, pA, conjA, α, β, backend)``: C = β C + α
    permutedims(op(A), linearize(pA)), on the device (the reference forwards
    this to StridedNative on the host)."""
    Cv, Av = _as_view(C), _as_view(A)
    perm = tuple(pA[0]) + tuple(pA[1])
    if sorted(perm) != list(range(1, Av.ndim + 1)) or len(perm) != Cv.ndim:
        raise ArgumentError("tensoradd: pA must be a permutation of A's axes with one entry per axis of C")
    indA = [0] * Av.ndim
    for i, ax in enumerate(perm):
        indA[ax - 1] = i + 1
    add_trace(Cv, alpha, Av, tuple(indA), beta, tuple(range(1, Cv.ndim + 1)), conjA=conjA)
    return C


def tensortrace(C, A, p, q, conjA, alpha, beta, backend: "QuasiStridedBackend" = None, allocator=None):
    """``TO.tensortrace!(C, A, p, q, conjA, α, β, backend)``: C = β C + α
    (partial trace of op(A) over the axis pairs (q[1][j], q[2][j]),
    remaining axes linearize(p) in C's order), on the device."""
    Cv, Av = _as_view(C), _as_view(A)
    keep_ax = tuple(p[0]) + tuple(p[1])
    q1, q2 = tuple(q[0]), tuple(q[1])
    if len(q1) != len(q2) or len(keep_ax) != Cv.ndim or \
            sorted(keep_ax + q1 + q2) != list(range(1, Av.ndim + 1)):
        raise ArgumentError("tensortrace: p and q must partition A's axes (q as pairs), p one per axis of C")
    indA = [0] * Av.ndim
    for i, ax in enumerate(keep_ax):
        indA[ax - 1] = i + 1
    for j, (x, y) in enumerate(zip(q1, q2)):
        indA[x - 1] = indA[y - 1] = -(j + 1)
    add_trace(Cv, alpha, Av, tuple(indA), beta, tuple(range(1, Cv.ndim + 1)), conjA=conjA)
    return C


def tensorcontract(C, A, pA, conjA, B, pB, conjB, pAB, alpha, beta,
                   backend: QuasiStridedBackend, allocator=None):
    """``TO.tensorcontract!(C, A, pA, conjA, B, pB, conjB, pAB, α, β, backend)``."""
    Cv = C if isinstance(C, StridedView) else StridedView(C)
    Av = A if isinstance(A, StridedView) else StridedView(A)
    Bv = B if isinstance(B, StridedView) else StridedView(B)
    if len(pA[0]) + len(pA[1]) != Av.ndim or len(pB[0]) + len(pB[1]) != Bv.ndim or \
            len(pAB[0]) + len(pAB[1]) != Cv.ndim:
        raise ArgumentError("invalid permutation of length")
    indA, indB, indC = contraction_labels(pA, pB, pAB)
    # dimcheck_tensorcontract: matching extents are checked by the planner.
    contract(Cv, alpha, Av, indA, Bv, indB, beta, indC, accumulator=backend.accumulator,
             conjA=conjA, conjB=conjB, allocator=allocator)
    return C
