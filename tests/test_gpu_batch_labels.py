"""Batch labels (QS_PLAN_BATCH_LABELS) on the device: every batch entry is
the contraction of that entry's sub-views, checked against the oracle run on
those sub-views in the plan's K order.  The gather GEMM (grid z over
entries), the skinny kernel, the scale path, the tensor-core methods (one
pass per entry), strided and negative-stride views, conj, alpha/beta
short-circuits, and the errors."""
import itertools

import numpy as np
import pytest
import torch

from _util import NP, Pair, colmajor_pair, randn, rel_fro
from oracle.oracle import HostView

pytestmark = pytest.mark.gpu


def entry_views(v: HostView, ind, blabels, bidx):
    """The sub-view of batch entry ``bidx`` (batch axes dropped)."""
    off = v.offset
    size, strides, keep = [], [], []
    for ax, l in enumerate(ind):
        if l in blabels:
            off += bidx[blabels.index(l)] * v.strides[ax]
        else:
            size.append(v.size[ax])
            strides.append(v.strides[ax])
            keep.append(l)
    return HostView(v.parent, tuple(size), tuple(strides), off, v.op), tuple(keep)


def oracle_batched(orc, C, alpha, A, indA, B, indB, beta, indC, blabels, extents, korder, **kw):
    """Runs the oracle on every batch entry of the host views in place."""
    for bidx in itertools.product(*[range(e) for e in extents]):
        a, ia = entry_views(A.host, indA, blabels, bidx)
        b, ib = entry_views(B.host, indB, blabels, bidx)
        c, ic = entry_views(C.host, indC, blabels, bidx)
        orc.brute(c, alpha, a, ia, b, ib, beta, ic, korder=list(korder) or None, **kw)


def run(qs, orc, C, alpha, A, indA, B, indB, beta, indC, blabels, extents, **kw):
    plan = qs.plan_contract(C.dev, A.dev, indA, B.dev, indB, indC, batch_labels=True, **kw)
    qs.execute(plan, alpha, beta)
    torch.cuda.synchronize()
    oracle_batched(orc, C, alpha, A, indA, B, indB, beta, indC, blabels, extents, plan.k_labels,
                   conjA=kw.get("conjA", False), conjB=kw.get("conjB", False))
    return C.device_parent(), C.host.parent, plan


@pytest.mark.parametrize("et", ["Float64", "Float32"])
@pytest.mark.parametrize("ab", [(1.0, 0.0), (1.5, -0.5)])
def test_batched_matmul_bitwise(qs, orc, et, ab):
    rng = np.random.default_rng(71)
    P, M, K, N = 7, 33, 20, 70
    A = colmajor_pair(qs, rng, (M, K, P), et)
    B = colmajor_pair(qs, rng, (K, N, P), et)
    C = colmajor_pair(qs, rng, (M, N, P), et, fill=np.nan if ab[1] == 0 else None)
    C0 = C.host.parent.copy()
    got, want, plan = run(qs, orc, C, ab[0], A, (1, 2, 9), B, (2, 3, 9), ab[1], (1, 3, 9), [9], [P],
                          method="native")
    assert plan.batch_length == P and plan.method == "native"
    eps = np.finfo(np.float64 if et == "Float64" else np.float32).eps
    assert rel_fro(got, want) <= 50 * K * eps   # Float64: the DMMA kernel over grid z
    if et == "Float64":
        # the SIMT tile keeps the ScalarKernel FMA order, per entry
        C.host.parent[:] = C0
        C.dev.parent.copy_(torch.from_numpy(C0))
        got, want, plan = run(qs, orc, C, ab[0], A, (1, 2, 9), B, (2, 3, 9), ab[1], (1, 3, 9), [9], [P],
                              method="native", native_tile=1)
        assert np.array_equal(got, want)


def test_two_batch_labels_strided_conj_complex(qs, orc):
    # batch labels in different positions of each operand; A a window of a
    # larger parent with a negative stride; conj on B.
    rng = np.random.default_rng(72)
    b1, b2, m, k, n = 3, 4, 17, 9, 21
    parent = randn(rng, 20000, "ComplexF64")
    # A[b1, m, b2, k] with strides chosen inside the parent, one negative
    A = Pair(qs, parent, (b1, m, b2, k), (1, -3, 60, 300), 3000)
    B = colmajor_pair(qs, rng, (k, b2, n, b1), "ComplexF64")
    C = colmajor_pair(qs, rng, (n, b1, m, b2), "ComplexF64")
    got, want, plan = run(qs, orc, C, 0.5 - 0.25j, A, (7, 1, 8, 2), B, (2, 8, 3, 7), 1.0 + 0.5j,
                          (3, 7, 1, 8), [7, 8], [b1, b2], conjB=True, method="native")
    assert sorted(plan.batch_labels) == [7, 8] and plan.batch_length == b1 * b2
    assert rel_fro(got, want) <= 50 * k * np.finfo(np.float64).eps


def test_batched_skinny_and_scale_paths(qs, orc):
    rng = np.random.default_rng(73)
    P, M, K, N = 5, 3000, 10, 12          # N <= 16, K <= 64: the skinny kernel
    A = colmajor_pair(qs, rng, (M, K, P), "Float64")
    B = colmajor_pair(qs, rng, (K, N, P), "Float64")
    C = colmajor_pair(qs, rng, (M, N, P), "Float64")
    got, want, _ = run(qs, orc, C, 2.0, A, (1, 2, 9), B, (2, 3, 9), 0.5, (1, 3, 9), [9], [P])
    assert np.array_equal(got, want)
    # alpha == 0: every entry of C scaled, A and B never read (NaN poison)
    An = colmajor_pair(qs, rng, (M, K, P), "Float64", fill=np.nan)
    C2 = colmajor_pair(qs, rng, (M, N, P), "Float64")
    c0 = C2.device_parent().copy()
    plan = qs.plan_contract(C2.dev, An.dev, (1, 2, 9), B.dev, (2, 3, 9), (1, 3, 9), batch_labels=True)
    qs.execute(plan, 0.0, 3.0)
    torch.cuda.synchronize()
    assert np.array_equal(C2.device_parent(), 3.0 * c0)


@pytest.mark.parametrize("method,et,tol", [("ozaki", "Float64", 1e-13), ("ozaki", "ComplexF64", 1e-13),
                                           ("bf16x3", "Float32", 1e-5)])
def test_batched_tensor_core_methods(qs, orc, method, et, tol):
    rng = np.random.default_rng(74)
    P, M, K, N = 3, 256, 320, 192
    A = colmajor_pair(qs, rng, (P, M, K), et)   # batch label first in A
    B = colmajor_pair(qs, rng, (K, N, P), et)
    C = colmajor_pair(qs, rng, (M, N, P), et, fill=np.nan)
    plan = qs.plan_contract(C.dev, A.dev, (9, 1, 2), B.dev, (2, 3, 9), (1, 3, 9), batch_labels=True,
                            method=method)
    assert plan.method == method
    qs.execute(plan, 1.0, 0.0)
    torch.cuda.synchronize()
    oracle_batched(orc, C, 1.0, A, (9, 1, 2), B, (2, 3, 9), 0.0, (1, 3, 9), [9], [P], (), precision=1)
    assert rel_fro(C.device_parent(), C.host.parent) <= tol


def test_batch_errors_on_the_device(qs):
    rng = np.random.default_rng(75)
    A = colmajor_pair(qs, rng, (4, 5, 3), "Float64")
    B = colmajor_pair(qs, rng, (5, 6, 3), "Float64")
    C = colmajor_pair(qs, rng, (4, 6, 3), "Float64")
    with pytest.raises(qs.ArgumentError, match="appears in indA, indB, and indC"):
        qs.plan_contract(C.dev, A.dev, (1, 2, 9), B.dev, (2, 3, 9), (1, 3, 9))
    plan = qs.plan_contract(C.dev, A.dev, (1, 2, 9), B.dev, (2, 3, 9), (1, 3, 9), batch_labels=True)
    with pytest.raises(qs.ArgumentError, match="batch labels cannot join a group"):
        qs.ContractGroup([plan])
    # C's parent one element short of the last batch entry: BoundsError, nothing written
    par = torch.full((4 * 6 * 3 - 1,), 5.0, dtype=torch.float64, device="cuda")
    Cs = qs.StridedView(par, (4, 6, 3), (1, 4, 24), 0)
    p2 = qs.plan_contract(Cs, A.dev, (1, 2, 9), B.dev, (2, 3, 9), (1, 3, 9), batch_labels=True)
    with pytest.raises(qs.BoundsError):
        qs.execute(p2, 1.0, 0.0)
    torch.cuda.synchronize()
    assert torch.all(par == 5.0)
    # contract! with batch labels
    Cc = colmajor_pair(qs, rng, (4, 6, 3), "Float64", fill=0.0)
    qs.contract(Cc.dev, 1.0, A.dev, (1, 2, 9), B.dev, (2, 3, 9), 0.0, (1, 3, 9), batch_labels=True)
    torch.cuda.synchronize()
    a = A.device_parent().reshape((4, 5, 3), order="F")
    b = B.device_parent().reshape((5, 6, 3), order="F")
    assert np.allclose(Cc.device_parent().reshape((4, 6, 3), order="F"), np.einsum("ikb,kjb->ijb", a, b),
                       rtol=1e-14, atol=1e-14)
