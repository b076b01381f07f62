"""Parity at the benchmark workloads' full sizes.

 * The permuted 4-index contraction C[a,b,c,d] = 1.3 sum_{e,f} A[a,e,b,f]
   B[f,c,e,d] + 0.7 C at a..d = 64, e = f = 48 (M = N = 4096, K = 2304):
   every one of the 16.8M elements of C against the oracle's FP64 nest, and a
   sample spread over all four indices of C (every 8th a, b, c, d) against
   the oracle in binary128.  Both value distributions (uniform[-1,1], and the
   same scaled by 2^U, U in [-20, 20], along a and d); the Ozaki path, the
   DMMA kernel, and Float32 operands (Ozaki with 4 digits).
 * The ComplexF64 MPS environment update at chi = 1024 (D_W = 5, d = 2):
   T1 = L*A, T2 = T1*W, out = T2*conj(A), each step checked on its own device
   inputs; the skinny step 2 on every element, steps 1 and 3 (planar Ozaki,
   conj on load in step 3) on samples spread over their free indices, in
   binary128.
 * 200 uneven blocks of the U(1) network step (the block generator's real
   size distribution) in one grouped launch, every block of C against the
   oracle, Float64 and Float32.

Tolerances: relative Frobenius error <= 1e-13 for Float64/ComplexF64 and
<= 1e-5 for Float32 (the stated targets).
"""
import importlib

import numpy as np
import pytest
import torch

import bench
from _util import Pair, colmajor_pair

pytestmark = pytest.mark.gpu
TOL64, TOL32 = 1e-13, 1e-5


def c1_run(qs, dist, dtype, method):
    A_h, B_h, C_h = bench.host_inputs(wide=dist == "wide")
    if dtype == "f32":
        A_h, B_h, C_h = (x.astype(np.float32) for x in (A_h, B_h, C_h))
    sa, sb, sc = bench.shapes()
    st = bench.colmajor_strides
    Av = qs.StridedView(torch.from_numpy(A_h).cuda(), sa, st(sa), 0)
    Bv = qs.StridedView(torch.from_numpy(B_h).cuda(), sb, st(sb), 0)
    Cv = qs.StridedView(torch.from_numpy(C_h).cuda(), sc, st(sc), 0)
    L = bench.LABELS
    plan = qs.plan_contract(Cv, Av, L["indA"], Bv, L["indB"], L["indC"], method=method)
    qs.execute(plan, bench.ALPHA, bench.BETA)
    torch.cuda.synchronize()
    qs.check_status(plan)
    got = Cv.parent.cpu().numpy()
    info = (plan.method, plan.ozaki_slices, plan.native_tile)
    plan.release()
    return got, (A_h, B_h, C_h), info


@pytest.mark.parametrize("dist", ["uniform", "wide"])
@pytest.mark.parametrize("method", ["ozaki", "native"])
def test_c1_full_size_float64(qs, orc, dist, method):
    got, (A_h, B_h, C_h), info = c1_run(qs, dist, "f64", method)
    assert info[0] == method
    if method == "native":
        assert info[2] >= 5  # the DMMA kernel
    acc = bench.c1_accuracy(orc, got, A_h, B_h, C_h)
    assert acc["elements"] == 4096 * 4096
    assert acc["rel_err"] <= TOL64, (info, acc)
    assert acc["rel_err_binary128"] <= TOL64, (info, acc)


@pytest.mark.parametrize("dist", ["uniform", "wide"])
def test_c1_full_size_float32(qs, orc, dist):
    # Float32 operands and C; the error is measured against FP64 arithmetic
    # on the same Float32 values.
    got, (A_h, B_h, C_h), info = c1_run(qs, dist, "f32", "auto")
    assert info[0] == "ozaki" and info[1] == 4
    acc = bench.c1_accuracy(orc, got, A_h, B_h, C_h)
    assert acc["rel_err"] <= TOL32, (info, acc)
    assert acc["rel_err_binary128"] <= TOL32, (info, acc)


def _device_host(qs, pair_like, shape):
    """A Pair whose host and device values are the device result `pair_like`."""
    st, acc = [], 1
    for s in shape:
        st.append(acc)
        acc *= s
    return Pair(qs, pair_like.device_parent(), shape, st)


def _check_sample(orc, C: Pair, alpha, A: Pair, la, B: Pair, lb, lc, picks, conjB=False):
    """The device result on the picked sub-view against the oracle in binary128."""
    Cs = orc.label_subview(orc.HostView(np.zeros_like(C.host.parent), C.host.size, C.host.strides), lc, picks)
    orc.brute(Cs, alpha, orc.label_subview(A.host, la, picks), la, orc.label_subview(B.host, lb, picks), lb,
              0.0, lc, conjB=conjB, precision=1, threads=orc.max_threads())
    gs = orc.HostView(C.device_parent(), Cs.size, Cs.strides, Cs.offset).to_array()
    return orc.rel_fro(gs, Cs.to_array())


def test_c2_mps_update_full_size(qs, orc):
    rng = np.random.default_rng(2024)
    chi, D, d = 1024, 5, 2
    L = colmajor_pair(qs, rng, (chi, D, chi), "ComplexF64")
    A = colmajor_pair(qs, rng, (chi, d, chi), "ComplexF64")
    W = colmajor_pair(qs, rng, (D, d, D, d), "ComplexF64")
    # labels: al=1, w=2, al'=3, s=4, be=5, w'=6, t=7, be'=8
    T1 = colmajor_pair(qs, rng, (D, chi, d, chi), "ComplexF64", fill=0)
    p1 = qs.plan_contract(T1.dev, L.dev, (1, 2, 3), A.dev, (1, 4, 5), (2, 3, 4, 5))
    assert p1.method == "ozaki"
    qs.execute(p1, 1, 0)
    torch.cuda.synchronize()
    err1 = _check_sample(orc, T1, 1.0, L, (1, 2, 3), A, (1, 4, 5), (2, 3, 4, 5),
                         {3: (0, 16, 64), 5: (7, 16, 64)})
    assert err1 <= TOL64, err1
    T1d = _device_host(qs, T1, (D, chi, d, chi))
    T2 = colmajor_pair(qs, rng, (chi, chi, D, d), "ComplexF64", fill=0)
    p2 = qs.plan_contract(T2.dev, T1d.dev, (2, 3, 4, 5), W.dev, (2, 4, 6, 7), (3, 5, 6, 7))
    qs.execute(p2, 1, 0)
    torch.cuda.synchronize()
    ref2 = orc.HostView(np.zeros_like(T2.host.parent), T2.host.size, T2.host.strides)
    orc.brute(ref2, 1.0, T1d.host, (2, 3, 4, 5), W.host, (2, 4, 6, 7), 0.0, (3, 5, 6, 7),
              korder=list(p2.k_labels), threads=orc.max_threads())
    err2 = orc.rel_fro(T2.device_parent(), ref2.parent)
    assert err2 <= TOL64, err2
    T2d = _device_host(qs, T2, (chi, chi, D, d))
    O = colmajor_pair(qs, rng, (chi, D, chi), "ComplexF64", fill=0)
    p3 = qs.plan_contract(O.dev, T2d.dev, (3, 5, 6, 7), A.dev, (3, 7, 8), (5, 6, 8), conjB=True)
    assert p3.method == "ozaki"
    qs.execute(p3, 1, 0)
    torch.cuda.synchronize()
    err3 = _check_sample(orc, O, 1.0, T2d, (3, 5, 6, 7), A, (3, 7, 8), (5, 6, 8),
                         {5: (3, 16, 64), 8: (5, 16, 64)}, conjB=True)
    assert err3 <= TOL64, err3
    for p in (p1, p2, p3):
        p.release()


@pytest.mark.parametrize("et", ["Float64", "Float32"])
def test_c3_every_block_of_200(qs, orc, et):
    wl = importlib.import_module(qs.__name__ + ".workloads")
    blocks = wl.u1_blocks(n=200, seed=0, cap=1 << 21)
    rng = np.random.default_rng(31)
    ops, plans = [], []
    for b in blocks:
        sa, la = b.a_shape_labels()
        sb, lb = b.b_shape_labels()
        sc, lc = b.c_shape_labels()
        A = colmajor_pair(qs, rng, sa, et)
        B = colmajor_pair(qs, rng, sb, et)
        C = colmajor_pair(qs, rng, sc, et)
        ops.append((A, la, B, lb, C, lc))
        plans.append(qs.plan_contract(C.dev, A.dev, la, B.dev, lb, lc))
    assert len({p.method for p in plans}) >= 2  # tensor-core and gather classes
    g = qs.ContractGroup(plans, mode="persistent")
    g.execute([1.1] * len(plans), [0.6] * len(plans))
    torch.cuda.synchronize()
    g.release()
    tol = TOL64 if et == "Float64" else TOL32
    worst = 0.0
    for (A, la, B, lb, C, lc), p in zip(ops, plans):
        f64 = lambda v: orc.HostView(v.parent.astype(np.float64), v.size, v.strides, v.offset)  # noqa: E731
        ref = f64(C.host)
        orc.nest_f64(ref, 1.1, f64(A.host), la, f64(B.host), lb, 0.6, lc)
        err = orc.rel_fro(C.device_parent().astype(np.float64), ref.parent)
        worst = max(worst, err)
        assert err <= tol, (p.method, p.m_length, p.n_length, p.k_length, err)
        p.release()
    print(f"c3 {et}: worst block error {worst:.3e} over {len(plans)} blocks")
