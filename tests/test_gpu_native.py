"""GPU parity of the gather ("native") kernels and the bandwidth paths against
the oracle, mirroring the reference's execution tests
(test/execution/test_execute.jl, test_nest.jl, test_mixed.jl, test_c_panel.jl,
test_dot.jl, test_outer.jl).  Every call goes through the C ABI.
"""
import json
import os

import numpy as np
import pytest
import torch

from _util import NP, Pair, colmajor_pair, randn, rel_fro, run_pair

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
ELTYPES = ["Float64", "Float32", "ComplexF64", "ComplexF32"]


def load(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


def eps(et):
    return float(np.finfo(NP[et]).eps)


def test_worked_fixture_exact(qs, orc):
    g = load("worked_fixture.json")
    rng = np.random.default_rng(0)
    A = Pair(qs, np.array(g["A"]), (3, 5, 2), (1, 3, 15))
    B = Pair(qs, np.array(g["B"]), (5, 4), (1, 5))
    C = colmajor_pair(qs, rng, (3, 4, 2), "Float64", fill=np.nan)
    plan = qs.plan_contract(C.dev, A.dev, g["indA"], B.dev, g["indB"], g["indC"], method="native")
    qs.execute(plan, 1.0, 0.0)
    assert C.device_parent().tolist() == g["Cref"]
    # permuted views: Ap[k,b,a] == A[a,k,b], Bp[n,k] == B[k,n]
    p = g["permuted"]
    Ap = qs.StridedView(A.dev.parent, (5, 2, 3), (3, 15, 1), 0)
    Bp = qs.StridedView(B.dev.parent, (4, 5), (5, 1), 0)
    C2 = colmajor_pair(qs, rng, (3, 4, 2), "Float64", fill=0.0)
    qs.contract(C2.dev, 1.0, Ap, p["indA"], Bp, p["indB"], 0.0, g["indC"])
    assert C2.device_parent().tolist() == g["Cref"]
    # nonzero view offsets on A and C
    o = g["offset"]
    A4 = qs.StridedView(torch.tensor(o["A4"], dtype=torch.float64, device="cuda"), (3, 5, 2), (1, 4, 20), 1)
    Cfull = torch.zeros(32, dtype=torch.float64, device="cuda")
    Cv = qs.StridedView(Cfull, (3, 4, 2), (1, 4, 16), 1)
    qs.contract(Cv, 1.0, A4, g["indA"], B.dev, g["indB"], 0.0, g["indC"])
    assert Cv.to_tensor().cpu().numpy().ravel(order="F").tolist() == o["Cref"]
    assert torch.all(Cfull.reshape(2, 4, 4)[:, :, 0] == 0)


def _scalar(rng, et):
    r = rng.random()
    if r < 0.1:
        return 0.0
    if r < 0.2:
        return 1.0
    v = rng.choice(np.arange(-3.0, 3.5, 0.5))
    if et.startswith("Complex"):
        return complex(v, rng.choice(np.arange(-3.0, 3.5, 0.5)))
    return float(v)


@pytest.mark.parametrize("et", ELTYPES)
def test_randomized_agreement_with_oracle(qs, orc, et):
    # test/execution/test_nest.jl:50-74: random M/K/N in 1:37, random alpha/beta
    # including the 0/1 shortcuts, random conjugation, NaN C when beta == 0.
    rng = np.random.default_rng(0x5A17D817)
    for _ in range(12):
        Ma, Ka, Na = (int(x) for x in rng.integers(1, 38, 3))
        conjA, conjB = bool(rng.integers(2)), bool(rng.integers(2))
        alpha, beta = _scalar(rng, et), _scalar(rng, et)
        A = colmajor_pair(qs, rng, (Ma, Ka), et)
        B = colmajor_pair(qs, rng, (Ka, Na), et)
        C = colmajor_pair(qs, rng, (Ma, Na), et, fill=np.nan if beta == 0 else None)
        got, ref, plan = run_pair(qs, orc, C, alpha, A, (1, 2), B, (2, 3), beta, (1, 3),
                                  conjA=conjA, conjB=conjB, method="native")
        assert np.all(np.isfinite(got))
        tol = 50 * max(Ka, 1) * eps(et)
        assert rel_fro(got, ref) <= tol, (Ma, Ka, Na, plan)


@pytest.mark.parametrize("tile", [1, 4])
def test_native_simt_f64_bitwise_equals_scalar_kernel_order(qs, orc, tile):
    # The SIMT gather kernel accumulates muladd(a, b, acc) ascending in the
    # plan's K order, like ScalarKernel: bitwise equal to the oracle.
    rng = np.random.default_rng(7)
    for (Ma, Ka, Na) in ((37, 29, 23), (130, 70, 65), (3072 // 16, 128, 80)):
        A = colmajor_pair(qs, rng, (Ma, Ka), "Float64")
        B = colmajor_pair(qs, rng, (Ka, Na), "Float64")
        C = colmajor_pair(qs, rng, (Ma, Na), "Float64")
        got, ref, plan = run_pair(qs, orc, C, 1.3, A, (1, 2), B, (2, 3), 0.7, (1, 3), method="native",
                                  native_tile=tile)
        assert plan.native_tile == tile
        assert np.array_equal(got, ref)


@pytest.mark.parametrize("MKN", [(600, 150, 8), (500, 77, 16), (700, 200, 29), (300, 64, 33),
                                 (257, 300, 17)])
@pytest.mark.parametrize("b_nfast", [False, True])
def test_native_narrow_n_tiles_bitwise(qs, orc, MKN, b_nfast):
    # The SIMT narrow-N tile shapes (256 x 16, 128 x 32) keep the ascending-K
    # muladd order: bitwise equal to the oracle, for B stored K-fast or N-fast.
    Ma, Ka, Na = MKN
    tile = 3 if Na <= 16 else 2 if Na <= 32 else 1
    rng = np.random.default_rng(Ma + Na)
    A = colmajor_pair(qs, rng, (Ma, Ka), "Float64")
    C = colmajor_pair(qs, rng, (Ma, Na), "Float64")
    if b_nfast:
        B = colmajor_pair(qs, rng, (Na, Ka), "Float64")
        got, ref, _ = run_pair(qs, orc, C, 1.3, A, (1, 2), B, (3, 2), 0.7, (1, 3), method="native",
                               native_tile=tile)
    else:
        B = colmajor_pair(qs, rng, (Ka, Na), "Float64")
        got, ref, _ = run_pair(qs, orc, C, 1.3, A, (1, 2), B, (2, 3), 0.7, (1, 3), method="native",
                               native_tile=tile)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("et", ["Float64", "ComplexF64", "Float32"])
@pytest.mark.parametrize("MKN", [(70000, 10, 10), (5000, 64, 16), (3000, 7, 3)])
def test_skinny_path(qs, orc, et, MKN):
    # N <= 16, K <= 64: one thread per row, B in shared memory; the
    # ScalarKernel FMA order, so real Float64 is bitwise equal to the oracle.
    M, K, N = MKN
    rng = np.random.default_rng(M + K + N)
    A = colmajor_pair(qs, rng, (M, K), et)
    B = colmajor_pair(qs, rng, (K, N), et)
    C = colmajor_pair(qs, rng, (M, N), et)
    got, ref, plan = run_pair(qs, orc, C, 1.3, A, (1, 2), B, (2, 3), 0.7, (1, 3), method="native")
    if et == "Float64":
        assert np.array_equal(got, ref)
    else:
        assert rel_fro(got, ref) <= 50 * K * eps(et)


def test_small_problem_tiles(qs, orc):
    # The c0 permuted matmul (M = (a,b) = 96*32, N = 80, K = 128).  Real
    # Float64 operands take the DMMA kernel with 64x64 tiles.  The SIMT kernel's 32x32
    # tiles (forced) keep the ScalarKernel FMA order: bitwise equal.
    rng = np.random.default_rng(96)
    A = colmajor_pair(qs, rng, (96, 128, 32), "Float64")
    B = colmajor_pair(qs, rng, (128, 80), "Float64")
    C = colmajor_pair(qs, rng, (96, 80, 32), "Float64")
    C0 = C.host.parent.copy()
    got, ref, plan = run_pair(qs, orc, C, 1.0, A, (1, 2, 3), B, (2, 4), 0.0, (1, 4, 3))
    assert plan.method == "native" and plan.native_tile == 4 + 2 + 1
    assert rel_fro(got, ref) <= 50 * 128 * eps("Float64")
    C.host.parent[:] = C0
    C.dev.parent.copy_(torch.from_numpy(C0))
    got, ref, plan = run_pair(qs, orc, C, 1.0, A, (1, 2, 3), B, (2, 4), 0.0, (1, 4, 3), native_tile=4)
    assert plan.method == "native" and plan.native_tile == 4
    assert np.array_equal(got, ref)


def test_permuted_zero_and_negative_strides_sliced_c(qs, orc):
    # test/execution/test_nest.jl:76-92
    rng = np.random.default_rng(11)
    a_n, k_n, b_n, n_n = 7, 11, 5, 9
    A = Pair(qs, randn(rng, a_n * k_n, "Float64"), (k_n, b_n, a_n), (a_n, 0, 1), 0)
    B = Pair(qs, randn(rng, k_n * n_n, "Float64"), (k_n, n_n), (-1, k_n), k_n - 1)
    big = randn(rng, (a_n + 2) * (n_n + 3) * (b_n + 1), "Float64")
    C = Pair(qs, big, (a_n, n_n, b_n), (1, a_n + 2, (a_n + 2) * (n_n + 3)), 1 + (a_n + 2))
    got, ref, _ = run_pair(qs, orc, C, 1.3, A, (2, 3, 1), B, (2, 4), 0.6, (1, 4, 3))
    assert rel_fro(got, ref) <= 50 * k_n * eps("Float64")
    # untouched padding of C's parent
    untouched = np.ones(big.size, dtype=bool)
    idx = np.add.outer(np.add.outer(np.arange(a_n), (a_n + 2) * np.arange(n_n)),
                       (a_n + 2) * (n_n + 3) * np.arange(b_n)) + 1 + (a_n + 2)
    untouched[idx.ravel()] = False
    assert np.array_equal(got[untouched], big[untouched])


def test_irregular_multilabel_m(qs, orc):
    # test/execution/test_nest.jl:94-110: M = (a, q), C padded along a.
    rng = np.random.default_rng(12)
    a_n, q_n, k_n, n_n = 7, 2, 5, 3
    A = colmajor_pair(qs, rng, (a_n, q_n, k_n), "Float64")
    B = colmajor_pair(qs, rng, (k_n, n_n), "Float64")
    C = Pair(qs, randn(rng, (a_n + 3) * q_n * n_n, "Float64"), (a_n, q_n, n_n),
             (1, a_n + 3, (a_n + 3) * q_n))
    got, ref, _ = run_pair(qs, orc, C, 1.7, A, (1, 2, 3), B, (3, 4), -0.4, (1, 2, 4))
    assert rel_fro(got, ref) <= 50 * k_n * eps("Float64")


@pytest.mark.parametrize("et", ["ComplexF64", "ComplexF32"])
def test_conjugation_sources_compose_by_xor(qs, orc, et):
    rng = np.random.default_rng(13)
    Am, Bm = randn(rng, 11 * 9, et), randn(rng, 9 * 7, et)
    for row in load("conj_xor.json"):
        A = Pair(qs, Am, (11, 9), (1, 11), 0, row["opA"])
        B = Pair(qs, Bm, (9, 7), (1, 9), 0, row["opB"])
        C = colmajor_pair(qs, rng, (11, 7), et, fill=0)
        qs.execute(qs.plan_contract(C.dev, A.dev, (1, 2), B.dev, (2, 3), (1, 3), conjA=row["conjA"]), 1, 0)
        got = C.device_parent().reshape(7, 11).T
        Ae = Am.reshape(9, 11).T
        Be = Bm.reshape(7, 9).T
        Ae = Ae.conj() if row["ca"] else Ae
        Be = Be.conj() if row["cb"] else Be
        assert np.allclose(got, Ae @ Be, rtol=50 * 9 * eps(et), atol=50 * 9 * eps(et))
        wrong = (Am.reshape(9, 11).T if row["ca"] else Am.reshape(9, 11).T.conj()) @ Be
        assert not np.allclose(got, wrong, rtol=50 * 9 * eps(et))


def test_short_circuits_and_empty_output(qs, orc):
    rng = np.random.default_rng(1)
    Ma, Na = 5, 4
    for Ka, alpha in ((0, 1.0), (6, 0.0)):
        for beta in (0.5, 0.0):
            A = colmajor_pair(qs, rng, (Ma, Ka), "Float64", fill=np.nan)
            B = colmajor_pair(qs, rng, (Ka, Na), "Float64", fill=np.nan)
            C = colmajor_pair(qs, rng, (Ma, Na), "Float64")
            C0 = C.host.parent.copy()
            plan = qs.plan_contract(C.dev, A.dev, (1, 2), B.dev, (2, 3), (1, 3))
            qs.execute(plan, alpha, beta)
            assert np.array_equal(C.device_parent(), beta * C0)
            if Ka == 0:
                assert plan.path == "ScalePath"
    # beta = 0 never reads a NaN C
    A = colmajor_pair(qs, rng, (11, 10), "Float64")
    B = colmajor_pair(qs, rng, (10, 9), "Float64")
    C = colmajor_pair(qs, rng, (11, 9), "Float64", fill=np.nan)
    got, ref, _ = run_pair(qs, orc, C, 2.5, A, (1, 2), B, (2, 3), 0.0, (1, 3))
    assert np.all(np.isfinite(got)) and rel_fro(got, ref) < 1e-14
    # empty M or N: a no-op
    for (M, N) in ((3, 0), (0, 3)):
        A = colmajor_pair(qs, rng, (M, 4), "Float64")
        B = colmajor_pair(qs, rng, (4, N), "Float64")
        C = colmajor_pair(qs, rng, (M, N), "Float64", fill=np.nan)
        before = C.device_parent().copy()
        plan = qs.plan_contract(C.dev, A.dev, (1, 2), B.dev, (2, 3), (1, 3))
        assert plan.path == "EmptyPath"
        qs.execute(plan, 1.0, 2.0)
        assert np.array_equal(C.device_parent(), before, equal_nan=True)


def test_out_of_bounds_rejected_before_any_write(qs):
    M, K, N = 8, 6, 5
    for sa, sb, sc in ((M * K - 1, K * N, M * N), (M * K, K * N - 1, M * N), (M * K, K * N, M * N - 1)):
        Cstore = torch.zeros(sc, dtype=torch.float64, device="cuda")
        A = qs.StridedView(torch.randn(sa, dtype=torch.float64, device="cuda"), (M, K), (1, M), 0)
        B = qs.StridedView(torch.randn(sb, dtype=torch.float64, device="cuda"), (K, N), (1, K), 0)
        plan = qs.plan_contract(qs.StridedView(Cstore, (M, N), (1, M), 0), A, (1, 2), B, (2, 3), (1, 3))
        with pytest.raises(qs.BoundsError):
            qs.execute(plan, 1.0, 0.0)
        torch.cuda.synchronize()
        assert torch.all(Cstore == 0)


MIXED = [
    ("Float32", "Float64", "Float64", None, (23, 37, 19), 0, False, False),
    ("Float64", "Float32", "Float32", None, (32, 40, 12), 1, False, False),
    ("Float64", "ComplexF64", "ComplexF64", None, (32, 32, 32), 0.3 - 0.7j, False, True),
    ("ComplexF32", "Float64", "ComplexF64", None, (32, 32, 32), 0.5, True, False),
    ("ComplexF32", "ComplexF64", "ComplexF64", None, (19, 29, 23), 1, True, True),
    ("Float64", "Float64", "ComplexF64", None, (18, 25, 14), 0.25 + 0.5j, False, False),
    ("ComplexF64", "Float32", "ComplexF64", "Float32", (17, 31, 13), 0, False, False),
    ("Float32", "Float64", "Float64", None, (1, 70, 29), 0.5, False, False),
    ("Float64", "Float32", "Float64", None, (37, 1, 21), 1, False, False),
]


@pytest.mark.parametrize("case", MIXED, ids=lambda c: f"{c[0]}x{c[1]}->{c[2]}")
def test_mixed_eltypes(qs, orc, case):
    # test/execution/test_mixed.jl:28-52: compute type, conversion on load,
    # one rounding on store; tolerance 10*sqrt(K)*eps in Frobenius norm.
    TA, TB, TC, acc, (M, K, N), beta, conjA, conjB = case
    rng = np.random.default_rng(7)
    A = colmajor_pair(qs, rng, (M, K), TA)
    B = colmajor_pair(qs, rng, (K, N), TB)
    C = colmajor_pair(qs, rng, (M, N), TC)
    got, ref, plan = run_pair(qs, orc, C, 1.5, A, (1, 2), B, (2, 3), beta, (1, 3),
                              conjA=conjA, conjB=conjB, accumulator=acc, precision=1)
    cdt = {"Float32": "Float32", "Float64": "Float64"}
    T = plan.compute_type
    rtol = 10 * np.sqrt(K) * max(eps("Float64" if "64" in T else "Float32"), eps(TC))
    assert rel_fro(got, ref) <= rtol, plan
    del cdt


@pytest.mark.parametrize("case", load("one_rounding.json"), ids=lambda c: f"{c['TC']}-{c['case']}")
def test_one_rounding_to_narrow_c(qs, case):
    M, N, K, beta = case["M"], case["N"], case["K"], case["beta"]
    A = np.zeros((M, K), dtype=NP[case["TA"]])
    A[:, 0] = 1
    A[:, K // 2] = 2.0 ** -30
    A[:, K - 1] = -1
    b = complex(*case["b"]) if case["TB"].startswith("Complex") else case["b"][0]
    TC = NP[case["TC"]]
    Av = qs.StridedView(torch.from_numpy(A.ravel(order="F").copy()).cuda(), (M, K), (1, M), 0)
    Bv = qs.StridedView(torch.from_numpy(np.full(K * N, b, dtype=NP[case["TB"]])).cuda(), (K, N), (1, K), 0)
    if case["case"] == "strided_c":
        parent = torch.from_numpy(np.zeros(2 * M * 3 * N, dtype=TC)).cuda()
        Cv = qs.StridedView(parent, (M, N), (2, 2 * M * 3), 1)
    else:
        parent = torch.from_numpy(np.zeros(M * N, dtype=TC)).cuda()
        Cv = qs.StridedView(parent, (M, N), (1, M), 0)
    fillv = np.nan if beta == 0 else 2.0 ** -28
    Cv.to_tensor()  # view sanity
    torch.as_strided(parent, Cv.size, Cv.strides, Cv.offset).fill_(fillv)
    plan = qs.plan_contract(Cv, Av, (1, 2), Bv, (2, 3), (1, 3), accumulator=case["accumulator"])
    qs.execute(plan, 1, beta)
    got = Cv.to_tensor().cpu().numpy()
    re, im = case["expected_re_im_before_rounding"]
    want = TC(complex(re, im)) if np.iscomplexobj(got) else TC(re)
    assert np.all(got == want)


@pytest.mark.parametrize("et", ELTYPES)
def test_dot_path(qs, orc, et):
    rng = np.random.default_rng(21)
    for (M, K, N) in ((1, 70, 29), (33, 300, 1), (1, 1000, 1)):
        A = colmajor_pair(qs, rng, (M, K), et)
        B = colmajor_pair(qs, rng, (K, N), et)
        C = colmajor_pair(qs, rng, (M, N), et)
        got, ref, plan = run_pair(qs, orc, C, 1.5, A, (1, 2), B, (2, 3), 0.5, (1, 3))
        assert plan.path == "DotPath"
        assert rel_fro(got, ref) <= 10 * np.sqrt(K) * eps(et)


@pytest.mark.parametrize("et", ELTYPES)
def test_outer_path(qs, orc, et):
    rng = np.random.default_rng(22)
    for beta in (0.0, 1.0, 0.5):
        A = colmajor_pair(qs, rng, (37,), et)
        B = colmajor_pair(qs, rng, (21,), et)
        C = colmajor_pair(qs, rng, (37, 21), et, fill=np.nan if beta == 0 else None)
        got, ref, plan = run_pair(qs, orc, C, 1.5, A, (1,), B, (2,), beta, (1, 2))
        assert plan.path == "OuterPath"
        assert rel_fro(got, ref) <= 4 * eps(et)


@pytest.mark.parametrize("et", ELTYPES)
def test_tensorcontract_edge_cases(qs, orc, et):
    # test/integrations/test_tensoroperations.jl:109-130
    rng = np.random.default_rng(13579)
    be = qs.QuasiStridedBackend()
    # outer product, conjA
    A = colmajor_pair(qs, rng, (3, 4), et)
    B = colmajor_pair(qs, rng, (5,), et)
    C = colmajor_pair(qs, rng, (5, 3, 4), et, fill=np.nan)
    qs.tensorcontract(C.dev, A.dev, ((1, 2), ()), True, B.dev, ((), (1,)), False, ((3, 1), (2,)), 1, 0, be)
    ref = np.einsum("ij,k->kij", np.conj(A.host.to_array()), B.host.to_array())
    assert rel_fro(C.device_parent().reshape(4, 3, 5).transpose(2, 1, 0), ref) <= 4 * eps(et)
    # full contraction to a scalar
    A = colmajor_pair(qs, rng, (3, 4), et)
    B = colmajor_pair(qs, rng, (4, 3), et)
    C = Pair(qs, np.full(1, np.nan, dtype=NP[et]), (), (), 0)
    qs.tensorcontract(C.dev, A.dev, ((), (1, 2)), False, B.dev, ((2, 1), ()), False, ((), ()), 1, 0, be)
    ref = np.einsum("ij,ji->", A.host.to_array(), B.host.to_array())
    assert abs(C.device_parent()[0] - ref) <= 1e2 * eps(et) * max(1, abs(ref))
    # strided views, conjB
    pa = randn(rng, 6 * 8, et)
    pb = randn(rng, 8 * 10, et)
    A = Pair(qs, pa, (3, 4), (2, 12), 0)
    B = Pair(qs, pb, (4, 5), (2, 16), 0)
    C = colmajor_pair(qs, rng, (3, 5), et, fill=np.nan)
    qs.tensorcontract(C.dev, A.dev, ((1,), (2,)), False, B.dev, ((1,), (2,)), True, ((1, 2), ()), 1, 0, be)
    ref = A.host.to_array() @ np.conj(B.host.to_array())
    assert rel_fro(C.device_parent().reshape(5, 3).T, ref) <= 40 * eps(et)


def test_tensorcontract_agrees_with_oracle(qs, orc):
    # test/integrations/test_tensoroperations.jl:21-42: both cases, every
    # eltype, conj flags and (alpha, beta) pairs, NaN C when beta == 0.
    rng = np.random.default_rng(1234567)
    cases = (((3, 20, 5, 3, 4), (4, 6, 20, 3), ((3, 1, 4), (2, 5)), ((3, 1), (4, 2)), ((3, 1, 4), (5, 2)),
              (3, 5, 3, 6, 3)),
             ((4, 5, 6), (3, 5, 6), ((1,), (2, 3)), ((2, 3), (1,)), ((2, 1), ()), (3, 4)))
    for et in ELTYPES:
        for szA, szB, pA, pB, pAB, szC in cases:
            indA, indB, indC = qs.contraction_labels(pA, pB, pAB)
            for conj in ((False, False), (True, True)) if et.startswith("Complex") else ((False, False),):
                for alpha, beta in ((1, 0), (0.6, 0), (0.6, 0.3)):
                    A = colmajor_pair(qs, rng, szA, et)
                    B = colmajor_pair(qs, rng, szB, et)
                    C = colmajor_pair(qs, rng, szC, et, fill=np.nan if beta == 0 else None)
                    qs.tensorcontract(C.dev, A.dev, pA, conj[0], B.dev, pB, conj[1], pAB, alpha, beta,
                                      qs.QuasiStridedBackend())
                    orc.brute(C.host, alpha, A.host, indA, B.host, indB, beta, indC,
                              conjA=conj[0], conjB=conj[1])
                    got = C.device_parent()
                    assert np.all(np.isfinite(got))
                    K = int(np.prod(szA)) // int(np.prod(szC[:1])) if False else 60
                    assert rel_fro(got, C.host.parent) <= 10 * np.sqrt(K) * eps(et)


def test_plan_reuse_is_repeatable(qs, orc):
    rng = np.random.default_rng(31)
    A = colmajor_pair(qs, rng, (40, 21), "Float64")
    B = colmajor_pair(qs, rng, (21, 30), "Float64")
    C = colmajor_pair(qs, rng, (40, 30), "Float64")
    plan = qs.plan_contract(C.dev, A.dev, (1, 2), B.dev, (2, 3), (1, 3))
    qs.execute(plan, 1.0, 0.0)
    first = C.device_parent().copy()
    C.dev.parent.fill_(float("nan"))
    qs.execute(plan, 1.0, 0.0)
    assert np.array_equal(C.device_parent(), first)
