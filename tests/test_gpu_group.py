"""GPU tests of grouped execution (qs_group_*): the uneven blocks of a
U(1)-symmetric step run as grouped persistent launches (and as CUDA graphs,
and sequentially) give exactly the results of one execute per plan — the
grouped kernels run the same tile code on the same packed operands — and
match the oracle within the stated tolerances.
"""
import importlib

import numpy as np
import pytest
import torch

from _util import Pair, colmajor_pair, randn, rel_fro

pytestmark = pytest.mark.gpu


def _workloads(qs):
    return importlib.import_module(qs.__name__ + ".workloads")


def col_strides(shape):
    st, acc = [], 1
    for s in shape:
        st.append(acc)
        acc *= s
    return tuple(st)


class BlockOps:
    """Operands of one block: host values, and two device copies of C (one
    for the group, one for per-plan executes)."""

    def __init__(self, qs, rng, blk, et):
        sa, la = blk.a_shape_labels()
        sb, lb = blk.b_shape_labels()
        sc, lc = blk.c_shape_labels()
        self.la, self.lb, self.lc = la, lb, lc
        self.A = Pair(qs, randn(rng, int(np.prod(sa)), et), sa, col_strides(sa))
        self.B = Pair(qs, randn(rng, int(np.prod(sb)), et), sb, col_strides(sb))
        c0 = randn(rng, int(np.prod(sc)), et)
        self.c0 = c0
        self.Cg = qs.StridedView(torch.from_numpy(c0.copy()).cuda(), sc, col_strides(sc))
        self.Cr = qs.StridedView(torch.from_numpy(c0.copy()).cuda(), sc, col_strides(sc))
        self.Ch = Pair(qs, c0.copy(), sc, col_strides(sc))


def make_blocks(qs, et, n, seed, cap):
    wl = _workloads(qs)
    blocks = wl.u1_blocks(n=n, seed=seed, cap=cap)
    rng = np.random.default_rng(seed + 100)
    return blocks, [BlockOps(qs, rng, b, et) for b in blocks]


@pytest.mark.parametrize("et", ["Float64", "Float32"])
@pytest.mark.parametrize("mode,graph", [("persistent", False), ("persistent", True),
                                        ("sequential", False), ("sequential", True)])
def test_group_equals_per_plan(qs, orc, et, mode, graph):
    blocks, ops = make_blocks(qs, et, n=24, seed=3, cap=1 << 20)
    gplans = [qs.plan_contract(o.Cg, o.A.dev, o.la, o.B.dev, o.lb, o.lc) for o in ops]
    rplans = [qs.plan_contract(o.Cr, o.A.dev, o.la, o.B.dev, o.lb, o.lc) for o in ops]
    methods = {p.method for p in gplans}
    assert "native" in methods and len(methods) >= 2, methods  # both classes present
    alphas = [1.0 + 0.01 * i for i in range(len(ops))]
    betas = [0.0 if i % 3 == 0 else 0.5 for i in range(len(ops))]
    g = qs.ContractGroup(gplans, mode=mode, graph=graph)
    for rep in range(2):  # second pass: accumulate on the first result, replay
        g.execute(alphas, betas)
        for p, a, b in zip(rplans, alphas, betas):
            qs.execute(p, a, b)
        torch.cuda.synchronize()
        for o in ops:
            got = o.Cg.parent.cpu().numpy()
            ref = o.Cr.parent.cpu().numpy()
            assert np.array_equal(got, ref)
    info = g.info()
    assert info["nplans"] == len(ops)
    if mode == "persistent":
        assert info["launches"] <= 2 * 5 + info["single_plans"] * 5, info
        assert info["native_plans"] + info["tc_plans"] + info["single_plans"] == len(ops)
    # Oracle check of a few blocks after both passes: C1 = a*AB + b*C0,
    # C2 = a*AB + b*C1.
    tol = 1e-13 if et == "Float64" else 1e-5
    for i in (0, 1, len(ops) - 1):
        o = ops[i]
        for _ in range(2):
            orc.brute(o.Ch.host, alphas[i], o.A.host, o.la, o.B.host, o.lb, betas[i], o.lc,
                      korder=list(gplans[i].k_labels) or None)
        got = o.Cg.parent.cpu().numpy()
        assert rel_fro(got, o.Ch.host.parent) <= tol, (i, rel_fro(got, o.Ch.host.parent))
    g.release()


def test_group_mixed_classes_and_edge_paths(qs, orc):
    # One group: Ozaki Float64, Ozaki ComplexF64 (1m), split-BF16 Float32,
    # native Float64 and ComplexF32, a dot-path plan, an alpha == 0 plan (scale
    # only), an empty plan, and an Ozaki plan with an Inf in A (fixup).
    rng = np.random.default_rng(11)
    cases = []

    def mm(M, K, N, et, inf=False):
        A = colmajor_pair(qs, rng, (M, K), et)
        if inf:
            A.dev.parent[5] = float("inf")
            A.host.parent[5] = np.inf
        B = colmajor_pair(qs, rng, (K, N), et)
        c0 = randn(rng, max(1, M * N), et)
        Cg = qs.StridedView(torch.from_numpy(c0.copy()).cuda(), (M, N), (1, M))
        Cr = qs.StridedView(torch.from_numpy(c0.copy()).cuda(), (M, N), (1, M))
        cases.append((A, B, Cg, Cr))

    mm(300, 200, 260, "Float64")
    mm(256, 128, 130, "ComplexF64")
    mm(384, 192, 300, "Float32")
    mm(70, 50, 40, "Float64")
    mm(33, 17, 45, "ComplexF32")
    mm(500, 300, 1, "Float64")          # dot path
    mm(200, 150, 140, "Float64")        # alpha = 0 below
    mm(0, 10, 20, "Float64")            # empty
    mm(260, 150, 300, "Float64", inf=True)
    alphas = [1.3, 0.5 - 0.25j, 2.0, 1.0, 1j, 0.9, 0.0, 1.0, 1.1]
    betas = [0.7, 0.25j, 0.0, 1.0, 0.5, 0.0, 0.3, 0.0, 0.5]
    # tensor-core methods forced for the first three (small shapes default
    # to the gather kernel); the rest take the defaults
    meth = ["ozaki", "ozaki", "bf16x3"] + ["auto"] * (len(cases) - 3)
    meth[-1] = "ozaki"
    gp = [qs.plan_contract(Cg, A.dev, (1, 2), B.dev, (2, 3), (1, 3), method=m)
          for (A, B, Cg, _), m in zip(cases, meth)]
    rp = [qs.plan_contract(Cr, A.dev, (1, 2), B.dev, (2, 3), (1, 3), method=m)
          for (A, B, _, Cr), m in zip(cases, meth)]
    assert gp[0].method == "ozaki" and gp[1].method == "ozaki" and gp[2].method == "bf16x3"
    for mode, graph in (("persistent", False), ("persistent", True)):
        for _, _, Cg, Cr in cases:
            Cg.parent.copy_(Cr.parent)
        g = qs.ContractGroup(gp, mode=mode, graph=graph)
        g.execute(alphas, betas)
        torch.cuda.synchronize()
        g.release()
        snapshot = [Cr.parent.clone() for _, _, _, Cr in cases]
        for p, a, b in zip(rp, alphas, betas):
            qs.execute(p, a, b)
        torch.cuda.synchronize()
        for i, (_, _, Cg, Cr) in enumerate(cases):
            got, ref = Cg.parent.cpu().numpy(), Cr.parent.cpu().numpy()
            assert np.array_equal(got, ref, equal_nan=True), (mode, graph, i)
        for (_, _, _, Cr), s in zip(cases, snapshot):
            Cr.parent.copy_(s)
    # The Inf row: that row of C is non-finite, the rest finite.
    A, B, Cg, _ = cases[-1]
    got = Cg.parent.cpu().numpy().reshape(300, 260).T
    assert not np.all(np.isfinite(got[5])) and np.all(np.isfinite(np.delete(got, 5, axis=0)))


def test_group_rejects_bad_input_before_any_write(qs):
    rng = np.random.default_rng(2)
    A = colmajor_pair(qs, rng, (64, 32), "Float64")
    B = colmajor_pair(qs, rng, (32, 16), "Float64")
    C1 = colmajor_pair(qs, rng, (64, 16), "Float64")
    C2 = colmajor_pair(qs, rng, (64, 16), "Float64")
    p1 = qs.plan_contract(C1.dev, A.dev, (1, 2), B.dev, (2, 3), (1, 3))
    p2 = qs.plan_contract(C2.dev, A.dev, (1, 2), B.dev, (2, 3), (1, 3))
    with pytest.raises(qs.ArgumentError):
        qs.ContractGroup([p1, p1])
    g = qs.ContractGroup([p1, p2])
    before = C1.dev.parent.clone()
    with pytest.raises(qs.ArgumentError):  # complex alpha for a real plan
        g.execute([1.0, 1j], [0.0, 0.0])
    torch.cuda.synchronize()
    assert torch.equal(C1.dev.parent, before)
    g.release()


@pytest.mark.parametrize("et,M,K,N", [("Float64", 300, 200, 260), ("Float32", 256, 130, 300),
                                      ("Float64", 40, 30, 20)])
def test_plan_cuda_graph_replay(qs, et, M, K, N):
    # execute! on a reused plan replays a captured graph: same results as the
    # plain launches, including after an alpha/beta change (re-capture).
    rng = np.random.default_rng(M + N)
    A = colmajor_pair(qs, rng, (M, K), et)
    B = colmajor_pair(qs, rng, (K, N), et)
    c0 = randn(rng, M * N, et)
    Cg = qs.StridedView(torch.from_numpy(c0.copy()).cuda(), (M, N), (1, M))
    Cr = qs.StridedView(torch.from_numpy(c0.copy()).cuda(), (M, N), (1, M))
    pg = qs.plan_contract(Cg, A.dev, (1, 2), B.dev, (2, 3), (1, 3), cuda_graph=True)
    pr = qs.plan_contract(Cr, A.dev, (1, 2), B.dev, (2, 3), (1, 3))
    for a, b in ((1.0, 0.5), (1.0, 0.5), (2.0, 0.25), (2.0, 0.25)):
        qs.execute(pg, a, b)
        qs.execute(pr, a, b)
        torch.cuda.synchronize()
        assert torch.equal(Cg.parent, Cr.parent)
