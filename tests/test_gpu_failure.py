"""Failure detection on the GPU without a fault.

Every barrier wait in the tensor-core GEMM kernels is bounded.  Here a plan's
wait limit is set to 1 ms with the producers held (they issue no operand
copies), so the MMA thread's first wait for an operand tile cannot complete
and runs out: the kernel must record QS_ETIMEOUT, stop without writing C,
drain what it issued (nothing) and release its tensor memory.  The test then
checks that the status reads back as DeviceTimeout, that C is untouched, that
the GPU still answers, and that the same plan computes the right result once
the hold is lifted.  No wait runs out with copies in flight, and nothing
traps or faults.  Each GEMM kernel variant is covered: the CTA-pair Ozaki
kernel, the one-SM fixed-schedule kernel, the runtime-schedule kernel (5
slices), the one-product-per-stage kernel and split BF16x3.
"""
import time

import numpy as np
import pytest
import torch

from _util import colmajor_pair, rel_fro

pytestmark = pytest.mark.gpu

VARIANTS = {
    "pair": dict(method="ozaki"),
    "single_sm": dict(method="ozaki", oz_single_sm=True),
    "runtime_schedule": dict(method="ozaki", ozaki_slices=5),
    "per_product": dict(method="ozaki", per_product_gemm=True),
    "bf16x3": dict(method="bf16x3"),
}


@pytest.mark.parametrize("variant", list(VARIANTS))
def test_wait_runs_out_then_plan_recovers(qs, orc, variant):
    kw = VARIANTS[variant]
    et = "Float32" if variant == "bf16x3" else "Float64"
    rng = np.random.default_rng(404)
    M, K, N = 640, 384, 512   # several tiles, so every CTA of the grid waits
    A = colmajor_pair(qs, rng, (M, K), et)
    B = colmajor_pair(qs, rng, (K, N), et)
    C = colmajor_pair(qs, rng, (M, N), et)
    before = C.device_parent().copy()
    plan = qs.plan_contract(C.dev, A.dev, (1, 2), B.dev, (2, 3), (1, 3), **kw)
    assert plan.method == kw["method"]
    qs.set_wait_limit(plan, 1_000_000, hold_loads=True)   # 1 ms, no operand copies
    t0 = time.perf_counter()
    qs.execute(plan, 1.3, 0.7)
    with pytest.raises(qs.DeviceTimeout):
        qs.check_status(plan)
    assert time.perf_counter() - t0 < 10.0
    assert np.array_equal(C.device_parent(), before)       # nothing written
    x = torch.arange(1000, dtype=torch.float64, device="cuda")
    assert float((x * 2).sum()) == 999000.0                  # the GPU still answers
    qs.check_status(plan)                                    # the status word was cleared
    # The hold lifted, the same plan is correct.
    qs.set_wait_limit(plan, 0, hold_loads=False)
    qs.execute(plan, 1.3, 0.7)
    qs.check_status(plan)
    torch.cuda.synchronize()
    got = C.device_parent()
    orc.brute(C.host, 1.3, A.host, (1, 2), B.host, (2, 3), 0.7, (1, 3), korder=list(plan.k_labels) or None,
              precision=1)
    tol = 1e-5 if et == "Float32" else (1e-10 if variant == "runtime_schedule" else 1e-13)
    assert rel_fro(got, C.host.parent) <= tol
    plan.release()


def test_wait_limit_with_a_captured_graph(qs, orc):
    # A plan replaying a captured graph re-captures after the limit changes.
    rng = np.random.default_rng(405)
    M, K, N = 512, 256, 384
    A = colmajor_pair(qs, rng, (M, K), "Float64")
    B = colmajor_pair(qs, rng, (K, N), "Float64")
    C = colmajor_pair(qs, rng, (M, N), "Float64", fill=0.0)
    plan = qs.plan_contract(C.dev, A.dev, (1, 2), B.dev, (2, 3), (1, 3), method="ozaki", cuda_graph=True)
    qs.execute(plan, 1.0, 0.0)
    qs.check_status(plan)
    ok = C.device_parent().copy()
    C.dev.parent.fill_(7.0)
    qs.set_wait_limit(plan, 1_000_000, hold_loads=True)
    qs.execute(plan, 1.0, 0.0)
    with pytest.raises(qs.DeviceTimeout):
        qs.check_status(plan)
    assert torch.all(C.dev.parent == 7.0)
    qs.set_wait_limit(plan, 0, hold_loads=False)
    qs.execute(plan, 1.0, 0.0)
    qs.check_status(plan)
    assert np.array_equal(C.device_parent(), ok)
    plan.release()
