"""GPU tests of the serving loop: a mixed stream of requests (Float32,
Float64, ComplexF64; tensor-core and gather paths; a resident operand) gives
each request the same result alone and in the mix, under a generous budget
and under a tight one that splits the stream into many ticks; results match
the oracle within the stated tolerances."""
import importlib

import numpy as np
import pytest
import torch

from oracle.oracle import HostView

pytestmark = pytest.mark.gpu


def modules(qs):
    return (importlib.import_module(qs.__name__ + ".serving"),
            importlib.import_module(qs.__name__ + ".workloads"))


def col_strides(shape):
    st, acc = [], 1
    for s in shape:
        st.append(acc)
        acc *= s
    return tuple(st)


def make_requests(sv, rng):
    """(requests, residents) — small shapes so the oracle stays cheap."""
    reqs = []

    def arr(shape, dt):
        n = int(np.prod(shape))
        if np.issubdtype(np.dtype(dt), np.complexfloating):
            v = (rng.standard_normal(n) + 1j * rng.standard_normal(n)) / np.sqrt(2)
        else:
            v = rng.standard_normal(n)
        return v.astype(dt).reshape(shape, order="F")

    res = {"env:f64": arr((160, 12, 20), np.float64)}
    # (shapeA, indA, shapeB, indB, indC, dtype, beta)
    cases = [
        ((96, 128, 32), (1, 2, 3), (128, 80), (2, 4), (1, 4, 3), np.float64, 0.0),       # permuted matmul, gather
        ((512, 384), (1, 2), (384, 400), (2, 3), (1, 3), np.float64, 0.5),                # Ozaki
        ((512, 256), (1, 2), (256, 600), (2, 3), (3, 1), np.float32, 0.0),                # BF16x3, C transposed
        ((400, 300), (1, 2), (300, 600), (2, 3), (1, 3), np.complex128, 0.5),             # Ozaki, complex
        ((12, 9, 7), (1, 2, 3), (7, 9, 11), (3, 2, 4), (4, 1), np.float32, 0.0),          # gather, 2 K labels
        ((30, 20, 10), (3, 1, 2), (10, 40), (2, 4), (1, 4, 3), np.complex128, 0.0),       # gather complex
        ((64, 64), (1, 2), (64, 1), (2, 3), (1, 3), np.float64, 0.0),                     # dot path
    ]
    for sa, la, sb, lb, lc, dt, beta in cases:
        A, B = arr(sa, dt), arr(sb, dt)
        dims = dict(zip(la, sa))
        dims.update(zip(lb, sb))
        sc = tuple(dims[l] for l in lc)
        r = sv.ContractRequest(A, la, B, lb, lc, alpha=1.25, beta=beta, dtype=dt,
                               C0=arr(sc, dt) if beta else None)
        reqs.append(r)
    # resident operand as A: C[w, n] = sum_{a,b} env[a, b, w] * B[a, b, n]
    B = arr((160, 12, 150), np.float64)
    reqs.append(sv.ContractRequest("env:f64", (1, 2, 3), B, (1, 2, 4), (3, 4), alpha=0.5, dtype=np.float64))
    return reqs, res


def clone(sv, r):
    return sv.ContractRequest(r.A, r.indA, r.B, r.indB, r.indC, alpha=r.alpha, beta=r.beta,
                              C0=None if r.C0 is None else r.C0.copy(), dtype=r.dtype)


def run(qs, sv, reqs, residents, budget, max_tick_requests=512):
    be = sv.DeviceBackend(qs)
    srv = sv.ContractionServer(be, hbm_budget_bytes=budget, max_tick_requests=max_tick_requests)
    for k, a in residents.items():
        srv.put_resident(k, a)
    for r in reqs:
        srv.submit(r)
    srv.drain()
    assert srv.peak_used <= budget
    return srv


@pytest.mark.parametrize("budget", [8 << 30, 24 << 20])
def test_alone_equals_in_mix(qs, orc, budget):
    sv, _ = modules(qs)
    rng = np.random.default_rng(42)
    reqs, residents = make_requests(sv, rng)
    mix = [clone(sv, r) for r in reqs]
    srv = run(qs, sv, mix, residents, budget)
    if budget < (1 << 30):
        assert srv.ticks_launched > 1  # the tight budget really split the stream
    for r, m in zip(reqs, mix):
        alone = clone(sv, r)
        run(qs, sv, [alone], residents, 8 << 30)
        assert m.error is None and alone.error is None
        assert np.array_equal(m.result, alone.result), r.indC
    # FP64 oracle on every request (its own error is far below the bounds)
    for r, m in zip(reqs, mix):
        A = residents[r.A] if isinstance(r.A, str) else r.A
        dt = np.dtype(r.dtype)
        Cshape = m.result.shape
        C = HostView((r.C0.copy() if r.C0 is not None else np.zeros(Cshape, dtype=dt)).ravel(order="F"),
                     Cshape, col_strides(Cshape))
        orc.brute(C, r.alpha, HostView(A.ravel(order="F"), A.shape, col_strides(A.shape)), r.indA,
                  HostView(r.B.ravel(order="F"), r.B.shape, col_strides(r.B.shape)), r.indB, r.beta, r.indC)
        ref = C.parent
        got = m.result.ravel(order="F")
        tol = 1e-5 if dt in (np.float32, np.complex64) else 1e-13
        err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        assert err <= tol, (r.indA, r.indB, dt, err)


def test_serving_stream_generator_and_replay(qs):
    # A short Poisson stream of the mixed families through the server: every
    # request completes without error, latencies are positive and ordered.
    sv, wl = modules(qs)
    pool_elems = 1 << 22
    pool = wl.pool_arrays(pool_elems, seed=3)
    specs, offsets, residents = wl.serving_stream(24, rate=2000.0, seed=5, pool_elems=pool_elems)
    be = sv.DeviceBackend(qs)
    srv = sv.ContractionServer(be, hbm_budget_bytes=16 << 30)
    for k, (shape, dt) in residents.items():
        srv.put_resident(k, wl.colmajor_view(pool[np.dtype(dt)], shape))
    reqs = []
    for sp in specs:
        buf = pool[np.dtype(sp["dtype"])]
        A = sp["resident"] or wl.colmajor_view(buf, sp["shapeA"])
        B = wl.colmajor_view(buf, sp["shapeB"], pool_elems - int(np.prod(sp["shapeB"])))
        reqs.append(sv.ContractRequest(A, sp["indA"], B, sp["indB"], sp["indC"], dtype=sp["dtype"]))
    srv.replay(reqs, offsets)
    st = srv.stats(reqs)
    assert st["errors"] == 0 and st["requests"] == 24
    assert 0 < st["p50_ms"] <= st["p99_ms"]
    assert all(np.all(np.isfinite(r.result)) for r in reqs)
