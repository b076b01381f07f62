"""The native Float64 GEMM on the FP64 tensor cores (DMMA) against the oracle.

The reference's Float64 kernels are FMA chains over K (ScalarKernel,
src/microkernels/steps.jl:27-36; SIMDKernel :73-106), and its tests bound the
native kernels by 50*K*eps (test/execution/test_nest.jl:50-74).  The f64
mma.sync of B200 adds each output's eight products in K order with one
rounding per product (an FMA chain), and the kernel feeds it K ascending in
the plan's order, so its results are bitwise equal to the oracle's
ScalarKernel-order evaluation; these tests assert exactly that.  The DMMA
kernel gathers A and B straight from their strided storage through the
offset tables, so every layout class is covered: A and B with the free or
the contracted axis unit-stride, permuted multi-label groups, ragged edges
on every tile shape, zero and negative strides, a Float32 C, the beta
cases, non-finite values, batch labels and grouped launches.
"""
import numpy as np
import pytest
import torch

from _util import Pair, colmajor_pair, randn, run_pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tile", [5, 6, 7, 8, 9])
@pytest.mark.parametrize("a_mfast,b_nfast", [(True, False), (False, True), (True, True), (False, False)])
def test_dmma_tiles_and_layouts(qs, orc, tile, a_mfast, b_nfast):
    rng = np.random.default_rng(100 * tile + 10 * a_mfast + b_nfast)
    M, K, N = 301, 83, 149   # ragged against every tile shape and the 16-wide K tile
    if a_mfast:
        A = colmajor_pair(qs, rng, (M, K), "Float64")
        la = (1, 2)
    else:
        A = colmajor_pair(qs, rng, (K, M), "Float64")
        la = (2, 1)
    if b_nfast:
        B = colmajor_pair(qs, rng, (N, K), "Float64")
        lb = (3, 2)
    else:
        B = colmajor_pair(qs, rng, (K, N), "Float64")
        lb = (2, 3)
    C = colmajor_pair(qs, rng, (M, N), "Float64")
    got, ref, plan = run_pair(qs, orc, C, 1.3, A, la, B, lb, 0.7, (1, 3), method="native", native_tile=tile)
    assert plan.native_tile == tile
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("beta", [0.0, 1.0, -0.6])
def test_dmma_beta_cases_and_float32_c(qs, orc, beta):
    rng = np.random.default_rng(5)
    M, K, N = 260, 140, 300
    A = colmajor_pair(qs, rng, (M, K), "Float64")
    B = colmajor_pair(qs, rng, (K, N), "Float64")
    C = colmajor_pair(qs, rng, (M, N), "Float64", fill=np.nan if beta == 0 else None)
    got, ref, plan = run_pair(qs, orc, C, 0.9, A, (1, 2), B, (2, 3), beta, (1, 3), method="native")
    assert plan.native_tile >= 5   # the DMMA kernel
    assert np.all(np.isfinite(got)) and np.array_equal(got, ref)
    # Float64 operands into a Float32 C: computed in Float64, rounded once
    C32 = colmajor_pair(qs, rng, (M, N), "Float32", fill=np.nan if beta == 0 else None)
    got, ref, plan = run_pair(qs, orc, C32, 0.9, A, (1, 2), B, (2, 3), beta, (1, 3), method="native")
    assert plan.native_tile >= 5 and plan.compute_type == "Float64"
    assert np.array_equal(got, ref)   # the same Float64 value, rounded once


def test_dmma_permuted_four_index(qs, orc):
    # C[a,b,c,d] = sum_{e,f} A[a,e,b,f] B[f,c,e,d]: every group is two labels
    # with a stride jump, A is M-fast and B K-fast (the permuted 4-index
    # contraction's layout, at 24^4 x 20^2).
    rng = np.random.default_rng(44)
    a = b = c = d = 24
    e = f = 20
    A = colmajor_pair(qs, rng, (a, e, b, f), "Float64")
    B = colmajor_pair(qs, rng, (f, c, e, d), "Float64")
    C = colmajor_pair(qs, rng, (a, b, c, d), "Float64")
    got, ref, plan = run_pair(qs, orc, C, 1.3, A, (1, 5, 2, 6), B, (6, 3, 5, 4), 0.7, (1, 2, 3, 4),
                              method="native")
    assert plan.native_tile >= 5
    assert np.array_equal(got, ref)


def test_dmma_zero_negative_strides_and_offsets(qs, orc):
    # test/execution/test_nest.jl:76-92 at a size that fills several tiles:
    # A broadcast along one free axis (stride 0), B read backwards along K.
    rng = np.random.default_rng(11)
    a_n, k_n, b_n, n_n = 70, 61, 5, 90
    A = Pair(qs, randn(rng, a_n * k_n, "Float64"), (k_n, b_n, a_n), (a_n, 0, 1), 0)
    B = Pair(qs, randn(rng, k_n * n_n, "Float64"), (k_n, n_n), (-1, k_n), k_n - 1)
    big = randn(rng, (a_n + 2) * (n_n + 3) * (b_n + 1), "Float64")
    C = Pair(qs, big, (a_n, n_n, b_n), (1, a_n + 2, (a_n + 2) * (n_n + 3)), 1 + (a_n + 2))
    got, ref, plan = run_pair(qs, orc, C, 1.3, A, (2, 3, 1), B, (2, 4), 0.6, (1, 4, 3), method="native")
    assert plan.native_tile >= 5
    assert np.array_equal(got, ref)
    idx = np.add.outer(np.add.outer(np.arange(a_n), (a_n + 2) * np.arange(n_n)),
                       (a_n + 2) * (n_n + 3) * np.arange(b_n)) + 1 + (a_n + 2)
    untouched = np.ones(big.size, dtype=bool)
    untouched[idx.ravel()] = False
    assert np.array_equal(got[untouched], big[untouched])


def test_dmma_propagates_nan_and_inf(qs, orc):
    rng = np.random.default_rng(9)
    M, K, N = 200, 64, 180
    pa = randn(rng, M * K, "Float64")
    pa[5 + M * 7] = np.inf      # row 5 of A
    pa[17 + M * 40] = np.nan    # row 17
    A = Pair(qs, pa, (M, K), (1, M))
    B = colmajor_pair(qs, rng, (K, N), "Float64")
    C = colmajor_pair(qs, rng, (M, N), "Float64")
    got, ref, plan = run_pair(qs, orc, C, 1.0, A, (1, 2), B, (2, 3), 0.5, (1, 3), method="native")
    g, r = got.reshape(N, M).T, ref.reshape(N, M).T
    assert np.array_equal(np.isnan(g), np.isnan(r)) and np.array_equal(np.isinf(g), np.isinf(r))
    fin = np.isfinite(r)
    assert np.array_equal(g[fin], r[fin])


def test_dmma_batched_entries(qs, orc):
    from test_gpu_batch_labels import run as run_batched
    rng = np.random.default_rng(71)
    P, M, K, N = 5, 150, 40, 130
    A = colmajor_pair(qs, rng, (M, K, P), "Float64")
    B = colmajor_pair(qs, rng, (K, N, P), "Float64")
    C = colmajor_pair(qs, rng, (M, N, P), "Float64")
    got, want, plan = run_batched(qs, orc, C, 1.5, A, (1, 2, 9), B, (2, 3, 9), -0.5, (1, 3, 9), [9], [P],
                                  method="native")
    assert plan.native_tile >= 5 and plan.batch_length == P
    assert np.array_equal(got, want)


def test_dmma_grouped_equals_single(qs, orc):
    # A grouped launch runs the same DMMA tile code on every problem (tile
    # shape by N); each result is bitwise equal to the plan's own execute and
    # to the oracle.
    rng = np.random.default_rng(3)
    shapes = [(300, 70, 200), (129, 33, 20), (512, 96, 64), (77, 130, 12), (260, 64, 150)]
    cases = []
    for (M, K, N) in shapes:
        A = colmajor_pair(qs, rng, (M, K), "Float64")
        B = colmajor_pair(qs, rng, (K, N), "Float64")
        Cg = colmajor_pair(qs, rng, (M, N), "Float64")
        Cr = Pair(qs, Cg.host.parent.copy(), (M, N), (1, M))
        cases.append((A, B, Cg, Cr, K))
    gp = [qs.plan_contract(Cg.dev, A.dev, (1, 2), B.dev, (2, 3), (1, 3), method="native")
          for A, B, Cg, _, _ in cases]
    rp = [qs.plan_contract(Cr.dev, A.dev, (1, 2), B.dev, (2, 3), (1, 3), method="native")
          for A, B, _, Cr, _ in cases]
    g = qs.ContractGroup(gp, mode="persistent")
    g.execute([1.1] * len(cases), [0.4] * len(cases))
    for p in rp:
        qs.execute(p, 1.1, 0.4)
    torch.cuda.synchronize()
    g.release()
    for (A, B, Cg, Cr, K) in cases:
        assert np.array_equal(Cg.device_parent(), Cr.device_parent())
        orc.brute(Cr.host, 1.1, A.host, (1, 2), B.host, (2, 3), 0.4, (1, 3),
                  korder=list(gp[0].k_labels) or None)
        assert np.array_equal(Cg.device_parent(), Cr.host.parent)
