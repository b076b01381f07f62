"""qs_contract_noalloc against the allocating entry point, on the GPU.

qs_contract_noalloc exists for callers that cannot allocate device memory
when they contract — a serving loop where cudaMalloc/cudaFree would
synchronize the device and stall other requests in flight, or a host whose
memory pool forbids raw allocations.  It keeps the gather kernels' offset
tables in one fixed-size static device array instead of a plan workspace.
This test calls it through the C ABI twice in a row, on two different
problems (so stale contents of the shared array would show), and compares
each result with plan_contract + execute on the same gather kernel.
"""
import ctypes

import numpy as np
import pytest
import torch

from _util import colmajor_pair, rel_fro

pytestmark = pytest.mark.gpu


def _noalloc(qs, C, alpha, A, indA, B, indB, beta, indC, conjA=False):
    keep = []
    cC, cA, cB = C._c(keep), A._c(keep), B._c(keep)
    lab = lambda ind: (ctypes.c_int64 * max(1, len(ind)))(*ind)  # noqa: E731
    iA, iB, iC = lab(indA), lab(indB), lab(indC)
    o = qs._abi.qs_plan_options()
    o.conjA = int(conjA)
    za, zb = complex(alpha), complex(beta)
    al = (ctypes.c_double * 2)(za.real, za.imag)
    be = (ctypes.c_double * 2)(zb.real, zb.imag)
    rc = qs._abi.lib().qs_contract_noalloc(ctypes.byref(cC), al, ctypes.byref(cA), iA, ctypes.byref(cB), iB,
                                           be, iC, ctypes.byref(o), torch.cuda.current_stream().cuda_stream)
    qs._abi.check(rc)


def _case(qs, rng, shapes, labels, et, alpha, beta, conjA=False):
    (sa, sb, sc), (iA, iB, iC) = shapes, labels
    A = colmajor_pair(qs, rng, sa, et)
    B = colmajor_pair(qs, rng, sb, et)
    C1 = colmajor_pair(qs, rng, sc, et)
    C2 = qs.StridedView(C1.dev.parent.clone(), C1.dev.size, C1.dev.strides, 0)
    plan = qs.plan_contract(C1.dev, A.dev, iA, B.dev, iB, iC, method="native", conjA=conjA)
    qs.execute(plan, alpha, beta)
    _noalloc(qs, C2, alpha, A.dev, iA, B.dev, iB, beta, iC, conjA=conjA)
    torch.cuda.synchronize()
    return C1.device_parent(), C2.parent.cpu().numpy(), plan.k_length


def test_noalloc_matches_allocating_entry_point_twice():
    from conftest import load_engine
    qs = load_engine()
    rng = np.random.default_rng(2026)
    eps64 = float(np.finfo(np.float64).eps)
    # 1) C[a,n,b] = A[a,k,b] B[k,n] in Float64 (M non-contiguous in C)
    ref, got, K = _case(qs, rng, ((96, 128, 8), (128, 80), (96, 80, 8)), ((1, 2, 3), (2, 4), (1, 4, 3)),
                        "Float64", 1.3, 0.7)
    assert rel_fro(got, ref) <= 50 * K * eps64
    # 2) a different problem right after: permuted ComplexF64 with conj(A)
    ref, got, K = _case(qs, rng, ((12, 9, 10, 7), (7, 11, 9, 6), (12, 10, 11, 6)),
                        ((1, 5, 2, 6), (6, 3, 5, 4), (1, 2, 3, 4)), "ComplexF64", 0.5 - 0.25j, 1.0,
                        conjA=True)
    assert rel_fro(got, ref) <= 50 * K * eps64


def test_noalloc_rejects_sizes_beyond_its_scratch():
    from conftest import load_engine
    qs = load_engine()
    big = qs.StridedView(torch.zeros(1, dtype=torch.float64, device="cuda"), (300000,), (0,), 0)
    v = qs.StridedView(torch.zeros(1, dtype=torch.float64, device="cuda"), (300000,), (0,), 0)
    C = qs.StridedView(torch.zeros(1, dtype=torch.float64, device="cuda"), (), (), 0)
    with pytest.raises(qs.ArgumentError, match="static scratch"):
        _noalloc(qs, C, 1.0, big, (1,), v, (1,), 0.0, ())


def test_noalloc_scale_dot_outer_paths():
    # The other paths the entry point serves, each against plan_contract +
    # execute on the same problem: alpha == 0 (C *= beta, A and B unread),
    # beta == 1 with alpha == 0 (nothing launched), an empty K (C *= beta),
    # a dot shape (M == 1) and an outer product (no K).
    from conftest import load_engine
    qs = load_engine()
    rng = np.random.default_rng(77)
    eps64 = float(np.finfo(np.float64).eps)
    mm = ((40, 30), (30, 20), (40, 20))
    for alpha, beta in ((0.0, 0.5), (0.0, 1.0), (0.0, 0.0)):
        ref, got, _ = _case(qs, rng, mm, ((1, 2), (2, 3), (1, 3)), "Float64", alpha, beta)
        assert np.array_equal(got, ref)
    ref, got, _ = _case(qs, rng, ((40, 0), (0, 20), (40, 20)), ((1, 2), (2, 3), (1, 3)), "Float64", 1.5, 0.5)
    assert np.array_equal(got, ref)
    ref, got, K = _case(qs, rng, ((1, 700), (700, 29), (1, 29)), ((1, 2), (2, 3), (1, 3)), "Float64", 1.5, 0.5)
    assert rel_fro(got, ref) <= 10 * np.sqrt(K) * eps64
    ref, got, _ = _case(qs, rng, ((37,), (21,), (37, 21)), ((1,), (2,), (1, 2)), "ComplexF64", 1.5, 0.5)
    assert rel_fro(got, ref) <= 4 * eps64
