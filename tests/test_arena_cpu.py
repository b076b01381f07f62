"""Device-arena bookkeeping on the host (no GPU): an arena over caller
memory with no CUDA device is pure bookkeeping (nothing to order), so the
bump/LIFO/checkpoint/reset rules can be checked here through the C ABI.
The pointers are never dereferenced."""
import ctypes

import pytest
import torch

pytestmark = pytest.mark.skipif(torch.cuda.is_available(),
                                reason="with a device the base must be device memory (covered by the GPU tests)")

BASE = 1 << 32          # 256-byte aligned; never dereferenced


def arena(qs, nbytes):
    lib = qs._abi.lib()
    h = ctypes.c_void_p()
    qs._abi.check(lib.qs_arena_create(ctypes.byref(h), BASE, nbytes))
    return lib, h


def alloc(qs, lib, h, n):
    p = ctypes.c_void_p()
    qs._abi.check(lib.qs_arena_alloc(h, n, ctypes.byref(p)))
    return p.value - BASE


def used(lib, h):
    u, pk, cap = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_size_t()
    w = ctypes.c_int64()
    lib.qs_arena_get_info(h, ctypes.byref(u), ctypes.byref(pk), ctypes.byref(cap), ctypes.byref(w))
    return u.value, pk.value, cap.value


def test_bump_lifo_and_reset(qs):
    lib, h = arena(qs, 4096)
    assert alloc(qs, lib, h, 100) == 0          # 256-byte blocks
    cp = lib.qs_arena_checkpoint(h)
    assert cp == 256
    assert alloc(qs, lib, h, 300) == 256        # rounds to 512
    assert alloc(qs, lib, h, 1) == 768
    assert used(lib, h) == (1024, 1024, 4096)
    # freeing a block under the top only marks it; freeing the top pops both
    qs._abi.check(lib.qs_arena_free(h, BASE + 256, 300, None))
    assert used(lib, h)[0] == 1024
    qs._abi.check(lib.qs_arena_free(h, BASE + 768, 1, None))
    assert used(lib, h)[0] == 256
    # reset to a checkpoint drops everything above it
    assert alloc(qs, lib, h, 1000) == 256
    qs._abi.check(lib.qs_arena_reset(h, cp, None))
    assert used(lib, h) == (256, 1280, 4096)
    # freeing a block a reset already reclaimed does nothing
    qs._abi.check(lib.qs_arena_free(h, BASE + 256, 1000, None))
    assert used(lib, h)[0] == 256
    lib.qs_arena_destroy(h)


def test_arena_errors(qs):
    lib, h = arena(qs, 1024)
    alloc(qs, lib, h, 512)
    with pytest.raises(qs.EngineError, match="exhausted"):
        alloc(qs, lib, h, 1024)
    assert used(lib, h)[0] == 512                # nothing changed
    with pytest.raises(qs.ArgumentError, match="does not belong"):
        qs._abi.check(lib.qs_arena_free(h, BASE + 4096, 1, None))
    alloc(qs, lib, h, 256)
    with pytest.raises(qs.ArgumentError, match="checkpoint"):
        qs._abi.check(lib.qs_arena_reset(h, 128, None))     # inside a block
    with pytest.raises(qs.ArgumentError, match="checkpoint"):
        qs._abi.check(lib.qs_arena_reset(h, 4096, None))    # above the top
    lib.qs_arena_destroy(h)
    h2 = ctypes.c_void_p()
    with pytest.raises(qs.ArgumentError, match="aligned"):
        qs._abi.check(lib.qs_arena_create(ctypes.byref(h2), BASE + 8, 1024))
