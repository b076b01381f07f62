"""Plan workspace and intermediates from caller allocators: the device arena
(TO.BufferAllocator's counterpart) and PyTorch's caching allocator.

Follows the reference's "explicit allocators serve the packed panels" test
(test/execution/test_workspace.jl:45-78): the same plan from the default
pool and from each allocator gives identical results, release hands the
blocks back, reset returns the arena to its checkpoint.  Also: exhaustion
fails before anything is written; memory reused after a reset while earlier
work may still run is ordered after it; intermediates of a contraction
chain come from the arena; grouped plans from an arena."""
import pytest
import torch

pytestmark = pytest.mark.gpu


def mm_views(qs, M, K, N, seed, dtype=torch.float64):
    g = torch.Generator(device="cuda").manual_seed(seed)
    A = torch.randn(M, K, dtype=dtype, device="cuda", generator=g)
    B = torch.randn(K, N, dtype=dtype, device="cuda", generator=g)
    C = torch.zeros(M, N, dtype=dtype, device="cuda")
    return A, B, C


def run_plan(qs, A, B, C, **kw):
    plan = qs.plan_contract(qs.StridedView(C), qs.StridedView(A), (1, 3), qs.StridedView(B), (3, 2),
                            (1, 2), **kw)
    qs.execute(plan, 1.5, 0.0)
    torch.cuda.synchronize()
    return plan


@pytest.mark.parametrize("method,shape", [("native", (19, 23, 17)), ("ozaki", (512, 384, 320)),
                                          ("bf16x3", (512, 384, 320))])
def test_allocators_serve_the_workspace(qs, method, shape):
    M, K, N = shape
    dtype = torch.float32 if method == "bf16x3" else torch.float64
    A, B, Cref = mm_views(qs, M, K, N, 1717, dtype)
    ref_plan = run_plan(qs, A, B, Cref, method=method)
    assert ref_plan.workspace_bytes > 0
    for allocator in (qs.DeviceArena(64 << 20), qs.TorchAllocator()):
        cp = qs.allocator_checkpoint(allocator)
        C = torch.full_like(Cref, float("nan"))
        plan = run_plan(qs, A, B, C, method=method, allocator=allocator)
        assert plan.method == ref_plan.method and plan.workspace_bytes == ref_plan.workspace_bytes
        assert torch.equal(C, Cref)
        if isinstance(allocator, qs.DeviceArena):
            assert allocator.info()["used"] >= plan.workspace_bytes
        else:
            assert allocator.live_blocks() > 0
        plan.release()
        qs.allocator_reset(allocator, cp)
        if isinstance(allocator, qs.DeviceArena):
            assert allocator.info()["used"] == cp == 0
            allocator.close()
        else:
            assert allocator.live_blocks() == 0


def test_arena_exhaustion_fails_before_any_write(qs):
    A, B, C = mm_views(qs, 600, 500, 400, 3)
    C.fill_(7.0)
    arena = qs.DeviceArena(4096)
    with pytest.raises(qs.EngineError, match="arena exhausted|allocator has no"):
        run_plan(qs, A, B, C, method="ozaki", allocator=arena)
    torch.cuda.synchronize()
    assert torch.all(C == 7.0)
    assert arena.info()["used"] == 0   # the failed plan handed back what it had


def test_reuse_after_reset_waits_for_earlier_work(qs):
    # A long contraction and a short one with different offset tables take
    # the same arena memory in turn, with no host synchronization between
    # calls; the arena must order each plan's table uploads after the kernels
    # that read the previous tables.
    arena = qs.DeviceArena(256 << 20)
    big = mm_views(qs, 2048, 2048, 2048, 11)
    small_src = [torch.randn(40, 30, 20, dtype=torch.float64, device="cuda") for _ in range(4)]
    outs = []
    for it in range(4):
        A, B, C = big
        qs.contract(qs.StridedView(C), 1.0, qs.StridedView(A), (1, 3), qs.StridedView(B), (3, 2), 0.0, (1, 2),
                    method="native", allocator=arena)
        big_out = C.clone()
        # permute-contract a 3-index tensor with a matrix: different geometry
        T = small_src[it]
        W = torch.randn(30, 25, dtype=torch.float64, device="cuda")
        R = torch.zeros(20, 25, 40, dtype=torch.float64, device="cuda")
        qs.contract(qs.StridedView(R), 1.0, qs.StridedView(T), (1, 3, 2), qs.StridedView(W), (3, 4), 0.0,
                    (2, 4, 1), method="native", allocator=arena)
        outs.append((big_out, R, torch.einsum("acb,cd->bda", T, W)))
    torch.cuda.synchronize()
    A, B, _ = big
    ref = A @ B
    for big_out, R, Rref in outs:
        assert torch.allclose(big_out, ref, rtol=1e-12, atol=1e-10)
        assert torch.allclose(R, Rref, rtol=1e-12, atol=1e-12)
    assert arena.info()["used"] == 0 and arena.info()["peak"] > 0


def test_chain_intermediates_from_the_arena(qs):
    # X[a, d] = sum_{b,c} A[a, b] B[b, c] D[c, d], the intermediate from
    # tensoralloc; per request: checkpoint, contract twice, free, reset.
    arena = qs.DeviceArena(32 << 20)
    peaks = []
    for req in range(3):
        g = torch.Generator(device="cuda").manual_seed(req)
        A = torch.randn(96, 80, dtype=torch.complex128, device="cuda", generator=g)
        B = torch.randn(80, 72, dtype=torch.complex128, device="cuda", generator=g)
        D = torch.randn(72, 64, dtype=torch.complex128, device="cuda", generator=g)
        cp = qs.allocator_checkpoint(arena)
        T = qs.tensoralloc((96, 72), torch.complex128, True, arena)
        assert T.data_ptr() % 256 == 0
        qs.contract(qs.StridedView(T), 1.0, qs.StridedView(A), (1, 2), qs.StridedView(B), (2, 3), 0.0, (1, 3),
                    allocator=arena)
        X = torch.zeros(96, 64, dtype=torch.complex128, device="cuda")
        qs.contract(qs.StridedView(X), 1.0, qs.StridedView(T), (1, 3), qs.StridedView(D), (3, 4), 0.0, (1, 4),
                    allocator=arena)
        qs.tensorfree(T, arena)
        assert arena.info()["used"] == cp   # T was the last block: popped
        qs.allocator_reset(arena, cp)
        torch.cuda.synchronize()
        assert torch.allclose(X, A @ B @ D, rtol=1e-12, atol=1e-10)
        peaks.append(arena.info()["peak"])
    assert peaks[0] == peaks[-1]   # the same memory serves every request


def test_grouped_plans_from_an_arena(qs):
    arena = qs.DeviceArena(128 << 20)
    plans, outs = [], []
    for i, (M, K, N) in enumerate([(64, 48, 32), (300, 200, 260), (512, 256, 384)]):
        A, B, C = mm_views(qs, M, K, N, 50 + i)
        plans.append(qs.plan_contract(qs.StridedView(C), qs.StridedView(A), (1, 3), qs.StridedView(B), (3, 2),
                                      (1, 2), allocator=arena))
        outs.append((A, B, C))
    g = qs.ContractGroup(plans, mode="persistent")
    g.execute([1.0] * 3, [0.0] * 3)
    g.release()
    for p in reversed(plans):
        p.release()
    torch.cuda.synchronize()
    for A, B, C in outs:
        assert torch.allclose(C, A @ B, rtol=1e-12, atol=1e-10)
    assert arena.info()["used"] == 0


def test_marked_free_keeps_its_stream_fence(qs):
    # A lower block freed on stream S1 is only marked; the top block freed on
    # an idle stream S2 then pops both.  The memory must not come back before
    # S1's work is done: qs_arena_alloc (a host-side tensoralloc) waits for it.
    arena = qs.DeviceArena(1 << 20)
    low = arena.alloc(4096)
    top = arena.alloc(4096)
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    with torch.cuda.stream(s1):
        torch.cuda._sleep(200_000_000)   # ~0.1 s of device time that "uses" `low`
        done = torch.cuda.Event()
        done.record(s1)
    arena.free(low, 4096, s1)
    assert arena.info()["used"] > 0      # marked, not popped
    arena.free(top, 4096, s2)
    assert arena.info()["used"] == 0     # popped together
    again = arena.alloc(4096)
    assert again == low
    assert done.query(), "arena handed back memory while S1's work was still running"
    assert arena.info()["waits"] >= 1
    arena.free(again, 4096)
    torch.cuda.synchronize()
    arena.close()
