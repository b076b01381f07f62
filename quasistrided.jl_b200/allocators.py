"""Device allocators for plan workspace and intermediates.

The reference's plans take their packed panels from a TensorOperations
allocator (src/execution/workspace.jl:98-123; ``allocator`` keyword of
plan_contract, src/planning/plan.jl:115-133), and its TO.tensorcontract!
brackets each call with allocator_checkpoint!/allocator_reset!
(src/integrations/tensoroperations.jl:84-86).  The device counterparts:

* ``None`` (TO.DefaultAllocator): the library's stream-ordered pool.
* ``DeviceArena``: TO.BufferAllocator on the device (qs_arena_*), a bump
  allocator over one device buffer with checkpoint/reset.  Planning from it
  needs no cudaMalloc, and ``contract`` with it returns as soon as the work is
  enqueued.
* ``TorchAllocator``: workspace from PyTorch's caching allocator, through the
  qs_allocator callbacks.

``tensoralloc``/``tensorfree``/``allocator_checkpoint``/``allocator_reset``
mirror the TensorOperations functions of the same names for device tensors.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import torch

from . import _abi


def _stream_ptr(stream) -> int:
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    return int(getattr(stream, "cuda_stream", stream) or 0)


class DeviceArena:
    """A device bump allocator (TO.BufferAllocator on the device).

    ``nbytes`` of device memory, taken from PyTorch's allocator once.  Blocks
    are 256-byte aligned.  ``free`` of the last block pops it; ``reset``
    drops everything above a ``checkpoint``.  Memory handed back by either
    is reused only after the work enqueued before it on ``stream`` has run.
    """

    def __init__(self, nbytes: int, device=None):
        if int(nbytes) <= 0:
            raise _abi.ArgumentError("DeviceArena needs a positive size")
        dev = torch.device("cuda", torch.cuda.current_device() if device is None else
                           torch.device(device).index or 0)
        self.device = dev
        self.buffer = torch.empty(int(nbytes), dtype=torch.uint8, device=dev)
        self._base = self.buffer.data_ptr()
        h = ctypes.c_void_p()
        with torch.cuda.device(dev):
            _abi.check(_abi.lib().qs_arena_create(ctypes.byref(h), self._base, int(nbytes)))
        self._h = h

    @property
    def handle(self) -> int:
        """Address of the arena's qs_allocator (for qs_plan_options.allocator)."""
        return _abi.lib().qs_arena_allocator(self._h)

    def checkpoint(self) -> int:
        return int(_abi.lib().qs_arena_checkpoint(self._h))

    def reset(self, checkpoint: int, stream=None) -> None:
        _abi.check(_abi.lib().qs_arena_reset(self._h, int(checkpoint), _stream_ptr(stream)))

    def alloc(self, nbytes: int) -> int:
        p = ctypes.c_void_p()
        _abi.check(_abi.lib().qs_arena_alloc(self._h, int(nbytes), ctypes.byref(p)))
        return int(p.value)

    def free(self, ptr: int, nbytes: int = 0, stream=None) -> None:
        _abi.check(_abi.lib().qs_arena_free(self._h, int(ptr), int(nbytes), _stream_ptr(stream)))

    def tensor(self, shape: Sequence[int], dtype: torch.dtype) -> torch.Tensor:
        """A tensor of ``shape`` whose storage is a block of the arena."""
        shape = tuple(int(s) for s in shape)
        n = 1
        for s in shape:
            n *= s
        nbytes = n * torch.empty((), dtype=dtype).element_size()
        off = self.alloc(nbytes) - self._base
        return self.buffer[off:off + nbytes].view(dtype).view(shape)

    def info(self) -> dict:
        used, peak, cap = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_size_t()
        waits = ctypes.c_int64()
        _abi.check(_abi.lib().qs_arena_get_info(self._h, ctypes.byref(used), ctypes.byref(peak),
                                                ctypes.byref(cap), ctypes.byref(waits)))
        return {"used": used.value, "peak": peak.value, "capacity": cap.value, "waits": waits.value}

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            _abi.lib().qs_arena_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TorchAllocator:
    """Plan workspace from PyTorch's caching allocator (qs_allocator callbacks).

    Each block is a uint8 tensor kept alive until the plan hands it back;
    a block whose last use was on a stream other than the one it was allocated
    on is recorded on that stream, so the caching allocator reuses it in order.
    """

    def __init__(self, device=None):
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else
                                   torch.device(device).index or 0)
        self._live: dict = {}
        self._alloc_cb = _abi.ALLOC_FN(self._alloc)
        self._free_cb = _abi.FREE_FN(self._free)
        self._struct = _abi.qs_allocator(None, self._alloc_cb, self._free_cb)

    @property
    def handle(self) -> int:
        return ctypes.addressof(self._struct)

    def _alloc(self, ctx, nbytes):
        try:
            t = torch.empty(max(int(nbytes), 1), dtype=torch.uint8, device=self.device)
        except Exception:
            return None
        self._live[t.data_ptr()] = t
        return t.data_ptr()

    def _free(self, ctx, ptr, nbytes, stream):
        t = self._live.pop(ptr, None)
        if t is None:
            return
        try:
            s = torch.cuda.ExternalStream(stream, device=self.device) if stream else \
                torch.cuda.default_stream(self.device)
            if s.cuda_stream != torch.cuda.current_stream(self.device).cuda_stream:
                t.record_stream(s)
        except Exception:
            torch.cuda.synchronize(self.device)

    def live_blocks(self) -> int:
        return len(self._live)


def allocator_handle(allocator) -> Optional[int]:
    """The qs_allocator pointer for qs_plan_options.allocator (None: the pool)."""
    if allocator is None or type(allocator).__name__ == "DefaultAllocator":
        return None
    if isinstance(allocator, (DeviceArena, TorchAllocator)):
        return allocator.handle
    raise _abi.ArgumentError(f"unsupported allocator {allocator!r}: use None, DeviceArena or TorchAllocator")


def tensoralloc(shape, dtype, istemp: bool = False, allocator=None) -> torch.Tensor:
    """``TO.tensoralloc``: a device tensor from ``allocator``."""
    if isinstance(allocator, DeviceArena):
        return allocator.tensor(shape, dtype)
    allocator_handle(allocator)  # validates
    return torch.empty(tuple(shape), dtype=dtype, device="cuda")


def tensorfree(t: torch.Tensor, allocator=None, stream=None) -> None:
    """``TO.tensorfree!``: hand ``t`` back (pops it when it is the arena's last block)."""
    if isinstance(allocator, DeviceArena):
        allocator.free(t.data_ptr(), t.numel() * t.element_size(), stream)


def allocator_checkpoint(allocator=None):
    """``TO.allocator_checkpoint!``."""
    return allocator.checkpoint() if isinstance(allocator, DeviceArena) else None


def allocator_reset(allocator, checkpoint, stream=None) -> None:
    """``TO.allocator_reset!``: reclaim everything allocated after ``checkpoint``."""
    if isinstance(allocator, DeviceArena):
        allocator.reset(checkpoint, stream)
