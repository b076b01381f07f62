"""GPU tests of the device tensoradd!/tensortrace! (qs_tensoradd_trace),
against numpy on the same host values: permutations and partial traces of
strided views (offsets, negative strides), all eltypes and mixed inputs,
conjugation, the alpha/beta short-circuits with NaN poison, and errors
raised before anything is written."""
import numpy as np
import pytest
import torch

from _util import NP, Pair, colmajor_pair, randn

pytestmark = pytest.mark.gpu


def host_array(pair):
    """The numpy array a Pair's view denotes (logical axes in order)."""
    v = pair.host
    idx = np.zeros(v.size, dtype=np.int64) + v.offset
    for d, (n, st) in enumerate(zip(v.size, v.strides)):
        sh = [1] * len(v.size)
        sh[d] = n
        idx = idx + (np.arange(n) * st).reshape(sh)
    return v.parent[idx]


def tol(et):
    return 1e-5 if et in ("Float32", "ComplexF32") else 1e-13


@pytest.mark.parametrize("et", ["Float64", "ComplexF64", "Float32", "ComplexF32"])
@pytest.mark.parametrize("ab", [(1.0, 0.0), (1.5, 0.5), (0.5 - 0.25j, 1.0)])
def test_tensoradd_permutation(qs, et, ab):
    alpha, beta = ab
    if not et.startswith("Complex") and (complex(alpha).imag or complex(beta).imag):
        pytest.skip("complex scalars need a complex eltype")
    rng = np.random.default_rng(hash(et) % 1000)
    A = colmajor_pair(qs, rng, (7, 5, 9, 4), et)
    C = colmajor_pair(qs, rng, (9, 7, 4, 5), et, fill=np.nan if beta == 0 else None)
    a0 = host_array(A)
    c0 = host_array(C).copy()
    qs.tensoradd(C.dev, A.dev, ((3, 1), (4, 2)), False, alpha, beta)
    torch.cuda.synchronize()
    want = alpha * np.transpose(a0, (2, 0, 3, 1)) + (beta * c0 if beta != 0 else 0)
    got = C.device_parent().reshape((9, 7, 4, 5), order="F")
    assert np.linalg.norm(got - want) <= tol(et) * np.linalg.norm(want)


def test_tensoradd_strided_views_conj_and_mixed(qs):
    # A: a strided window with an offset and a negative stride, complex with
    # op conj XOR conjA; C: a sliced view of a larger parent.
    rng = np.random.default_rng(3)
    parent = randn(rng, 2000, "ComplexF64")
    A = Pair(qs, parent, (6, 8), (-3, 30), 300, op="conj")
    cpar = randn(rng, 400, "ComplexF64")
    C = Pair(qs, cpar, (8, 6), (1, 20), 7)
    a0 = host_array(A)
    c0 = host_array(C).copy()
    qs.tensoradd(C.dev, A.dev, ((2,), (1,)), True, 2.0, 0.5)  # conj(conj(A)) = A
    torch.cuda.synchronize()
    got_par = C.device_parent()
    idx = 7 + np.arange(8)[:, None] * 1 + np.arange(6)[None, :] * 20
    want = 2.0 * a0.T + 0.5 * c0
    assert np.linalg.norm(got_par[idx] - want) <= 1e-14 * np.linalg.norm(want)
    # everything outside the view is untouched
    mask = np.ones(400, bool)
    mask[idx.ravel()] = False
    assert np.array_equal(got_par[mask], cpar[mask])
    # Float32 A into Float64 C: converted on load
    A32 = colmajor_pair(qs, rng, (5, 6), "Float32")
    C64 = colmajor_pair(qs, rng, (6, 5), "Float64", fill=0.0)
    qs.tensoradd(C64.dev, A32.dev, ((2, 1), ()), False, 1.0, 0.0)
    torch.cuda.synchronize()
    assert np.array_equal(C64.device_parent().reshape((6, 5), order="F"),
                          host_array(A32).astype(np.float64).T)


@pytest.mark.parametrize("et", ["Float64", "ComplexF64"])
def test_tensortrace_partial_and_full(qs, et):
    rng = np.random.default_rng(5)
    A = colmajor_pair(qs, rng, (6, 7, 5, 7), et)
    a0 = host_array(A)
    # C[a, c] = sum_b A[a, b, c, b]
    C = colmajor_pair(qs, rng, (6, 5), et)
    c0 = host_array(C).copy()
    qs.tensortrace(C.dev, A.dev, ((1, 3), ()), ((2,), (4,)), False, 1.25, 0.5)
    torch.cuda.synchronize()
    want = 1.25 * np.einsum("abcb->ac", a0) + 0.5 * c0
    got = C.device_parent().reshape((6, 5), order="F")
    assert np.linalg.norm(got - want) <= 1e-13 * np.linalg.norm(want)
    # two traced pairs down to a scalar: sum_{i,j} B[i, j, i, j]
    B = colmajor_pair(qs, rng, (4, 3, 4, 3), et)
    S = colmajor_pair(qs, rng, (), et, fill=0)
    qs.tensortrace(S.dev, B.dev, ((), ()), ((1, 2), (3, 4)), True, 1.0, 0.0)
    torch.cuda.synchronize()
    want = np.conj(np.einsum("ijij->", host_array(B)))
    assert abs(S.device_parent()[0] - want) <= 1e-13 * abs(want)


def test_short_circuits_and_errors_before_any_write(qs):
    rng = np.random.default_rng(7)
    # alpha == 0: A is never read (NaN poison), C = beta * C
    A = colmajor_pair(qs, rng, (4, 5), "Float64", fill=np.nan)
    C = colmajor_pair(qs, rng, (5, 4), "Float64")
    c0 = C.device_parent().copy()
    qs.tensoradd(C.dev, A.dev, ((2, 1), ()), False, 0.0, 2.0)
    torch.cuda.synchronize()
    assert np.array_equal(C.device_parent(), 2.0 * c0)
    # beta == 0: C is never read (NaN poison)
    A2 = colmajor_pair(qs, rng, (4, 5), "Float64")
    C2 = colmajor_pair(qs, rng, (5, 4), "Float64", fill=np.nan)
    qs.tensoradd(C2.dev, A2.dev, ((2, 1), ()), False, 1.0, 0.0)
    torch.cuda.synchronize()
    assert np.all(np.isfinite(C2.device_parent()))
    before = C.device_parent().copy()
    with pytest.raises(qs.DimensionMismatch):       # extents differ
        bad = colmajor_pair(qs, rng, (4, 4), "Float64")
        qs.tensoradd(bad.dev, A2.dev, ((2, 1), ()), False, 1.0, 0.0)
    with pytest.raises(qs.ArgumentError):            # a C label missing from A
        qs.add_trace(C.dev, 1.0, A2.dev, (3, 1), 0.0, (1, 2))
    C1 = colmajor_pair(qs, rng, (5,), "Float64")
    with pytest.raises(qs.ArgumentError):            # an A label neither in C nor paired
        qs.add_trace(C1.dev, 1.0, A2.dev, (3, 1), 0.0, (1,))
    par = torch.zeros(10, dtype=torch.float64, device="cuda")
    oob = qs.StridedView(par, (5, 4), (1, 5), 0)     # needs 20 elements
    with pytest.raises(qs.BoundsError):
        qs.tensoradd(oob, A2.dev, ((2, 1), ()), False, 1.0, 0.0)
    torch.cuda.synchronize()
    assert np.array_equal(C.device_parent(), before) and torch.count_nonzero(par) == 0
