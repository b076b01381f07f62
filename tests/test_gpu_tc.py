"""GPU parity of the tensor-core paths: Float64 through INT8 Ozaki slices
(tcgen05 kind::i8) and Float32 through split-BF16 x3 (kind::f16), against the
oracle evaluated in binary128.  Tolerances are the stated targets:
relative Frobenius error <= 1e-13 (Float64), <= 1e-5 (Float32).
"""
import numpy as np
import pytest
import torch

from _util import Pair, colmajor_pair, rel_fro, run_pair

pytestmark = pytest.mark.gpu
TOL64, TOL32 = 1e-13, 1e-5


def uniform_pair(qs, rng, shape, et="Float64", scale_axis=None):
    n = int(np.prod(shape))
    v = rng.uniform(-1.0, 1.0, n)
    if scale_axis is not None:
        arr = v.reshape(shape, order="F")
        u = np.exp2(rng.integers(-20, 21, shape[scale_axis]).astype(np.float64))
        sh = [1] * len(shape)
        sh[scale_axis] = shape[scale_axis]
        v = (arr * u.reshape(sh)).ravel(order="F")
    st, acc = [], 1
    for s in shape:
        st.append(acc)
        acc *= s
    return Pair(qs, v.astype(np.float64 if et == "Float64" else np.float32), tuple(shape), tuple(st))


@pytest.mark.parametrize("MKN", [(256, 300, 384), (200, 333, 130), (128, 64, 128), (1000, 129, 777)])
@pytest.mark.parametrize("beta", [0.0, 1.0, 0.7])
@pytest.mark.parametrize("per_product", [False, True])
def test_ozaki_matmul_matches_oracle(qs, orc, MKN, beta, per_product):
    # Both GEMM kernels: grouped diagonals (default) and one product per stage.
    M, K, N = MKN
    rng = np.random.default_rng(M * 7 + K)
    A = uniform_pair(qs, rng, (M, K))
    B = uniform_pair(qs, rng, (K, N))
    C = colmajor_pair(qs, rng, (M, N), "Float64", fill=np.nan if beta == 0 else None)
    got, ref, plan = run_pair(qs, orc, C, 1.3, A, (1, 2), B, (2, 3), beta, (1, 3), method="ozaki",
                              precision=1, per_product_gemm=per_product)
    assert plan.method == "ozaki" and plan.ozaki_slices >= 6
    assert np.all(np.isfinite(got))
    assert rel_fro(got, ref) <= TOL64, rel_fro(got, ref)


def test_ozaki_is_the_default_for_float64(qs):
    # Past M*N*K = 2^26 the default is the Ozaki path; below it (and for
    # N < 64) the single-launch gather kernel.
    rng = np.random.default_rng(0)
    A = uniform_pair(qs, rng, (512, 512))
    B = uniform_pair(qs, rng, (512, 512))
    C = colmajor_pair(qs, rng, (512, 512), "Float64")
    assert qs.plan_contract(C.dev, A.dev, (1, 2), B.dev, (2, 3), (1, 3)).method == "ozaki"
    A2 = uniform_pair(qs, rng, (300, 200))
    B2 = uniform_pair(qs, rng, (200, 260))
    C2 = colmajor_pair(qs, rng, (300, 260), "Float64")
    assert qs.plan_contract(C2.dev, A2.dev, (1, 2), B2.dev, (2, 3), (1, 3)).method == "native"


@pytest.mark.parametrize("wide", [False, True])
def test_ozaki_permuted_4index(qs, orc, wide):
    # C[a,b,c,d] = sum_{e,f} A[a,e,b,f] * B[f,c,e,d] at a=b=c=d=32, e=f=24,
    # with the wide-exponent distribution scaling A along a and B along d.
    rng = np.random.default_rng(5 + wide)
    A = uniform_pair(qs, rng, (32, 24, 32, 24), scale_axis=0 if wide else None)
    B = uniform_pair(qs, rng, (24, 32, 24, 32), scale_axis=3 if wide else None)
    C = colmajor_pair(qs, rng, (32, 32, 32, 32), "Float64")
    got, ref, plan = run_pair(qs, orc, C, 1.3, A, (1, 5, 2, 6), B, (6, 3, 5, 4), 0.7, (1, 2, 3, 4),
                              method="ozaki", precision=1)
    assert plan.method == "ozaki"
    assert rel_fro(got, ref) <= TOL64, rel_fro(got, ref)


@pytest.mark.parametrize("et,tol", [("Float64", TOL64), ("Float32", TOL32)])
def test_ozaki_unit_stride_on_a_later_row_label(qs, orc, et, tol):
    # C[x,y,n1,n2] = sum_k A[y,k,x] B[n2,k,n1]: the M labels are (x, y) and
    # the N labels (n1, n2) in C's order, K is k; A is unit-stride along y
    # and B along n2, neither along its first row label nor along K, so the
    # pack visits their rows in the order with that label fastest.  Both
    # operands scaled by 2^U along a row label to vary the row exponents.
    rng = np.random.default_rng(17)
    x, y, k, n1, n2 = 24, 40, 150, 20, 16
    A = uniform_pair(qs, rng, (y, k, x), et, scale_axis=2)
    B = uniform_pair(qs, rng, (n2, k, n1), et, scale_axis=0)
    C = colmajor_pair(qs, rng, (x, y, n1, n2), et)
    got, ref, plan = run_pair(qs, orc, C, 1.3, A, (2, 5, 1), B, (4, 5, 3), 0.7, (1, 2, 3, 4),
                              method="ozaki", precision=1)
    assert plan.method == "ozaki" and plan.m_labels == (1, 2) and plan.n_labels == (3, 4)
    assert rel_fro(got, ref) <= tol, rel_fro(got, ref)


def test_ozaki_persistent_tiles_and_reuse(qs, orc):
    # 16 x 16 = 256 tiles > SM count: every CTA runs more than one tile.
    rng = np.random.default_rng(9)
    M = N = 2048
    K = 256
    A = uniform_pair(qs, rng, (M, K))
    B = uniform_pair(qs, rng, (K, N))
    C = colmajor_pair(qs, rng, (M, N), "Float64", fill=0.0)
    plan = qs.plan_contract(C.dev, A.dev, (1, 2), B.dev, (2, 3), (1, 3), method="ozaki")
    qs.execute(plan, 1.0, 0.0)
    first = C.device_parent().copy()
    sample = (0, 4 * M + 17)
    orc.brute(C.host, 1.0, A.host, (1, 2), B.host, (2, 3), 0.0, (1, 3), c_range=sample, precision=1)
    assert rel_fro(first[:sample[1]], C.host.parent[:sample[1]]) <= TOL64
    # last columns (last tiles of the schedule)
    lo = (N - 3) * M
    orc.brute(C.host, 1.0, A.host, (1, 2), B.host, (2, 3), 0.0, (1, 3), c_range=(lo, N * M), precision=1)
    assert rel_fro(first[lo:], C.host.parent[lo:]) <= TOL64
    C.dev.parent.fill_(float("nan"))
    qs.execute(plan, 1.0, 0.0)
    assert np.array_equal(C.device_parent(), first)


@pytest.mark.parametrize("slices", [0, 8])
def test_ozaki_long_k_segments(qs, orc, slices):
    # K beyond one INT32-exact segment (148 K blocks at 7 slices); slices=0
    # takes the default for this K (7, the fixed-schedule kernel).
    rng = np.random.default_rng(10)
    M, K, N = 128, 20000, 128
    A = uniform_pair(qs, rng, (M, K))
    B = uniform_pair(qs, rng, (K, N))
    C = colmajor_pair(qs, rng, (M, N), "Float64")
    got, ref, plan = run_pair(qs, orc, C, 1.0, A, (1, 2), B, (2, 3), 0.5, (1, 3), method="ozaki",
                              ozaki_slices=slices, precision=1)
    assert plan.ozaki_slices == (7 if slices == 0 else slices)
    assert rel_fro(got, ref) <= TOL64, rel_fro(got, ref)


@pytest.mark.parametrize("slices,tol", [(5, 1e-10), (6, TOL64), (7, TOL64)])
def test_ozaki_slice_counts(qs, orc, slices, tol):
    # Each schedule: s = 5 ({0}, {1..4}), 6 ({0, 1}, {2..5}), 7 ({0..2}, {3..6});
    # 5 slices are below the 1e-13 target and checked at their own accuracy.
    rng = np.random.default_rng(20 + slices)
    M, K, N = 300, 500, 260
    A = uniform_pair(qs, rng, (M, K))
    B = uniform_pair(qs, rng, (K, N))
    C = colmajor_pair(qs, rng, (M, N), "Float64")
    got, ref, plan = run_pair(qs, orc, C, 1.3, A, (1, 2), B, (2, 3), 0.7, (1, 3), method="ozaki",
                              ozaki_slices=slices, precision=1)
    assert plan.ozaki_slices == slices
    assert rel_fro(got, ref) <= tol, rel_fro(got, ref)


def test_ozaki_nonfinite_rows_and_columns(qs, orc):
    # NaN/Inf in a row of A or a column of B: those elements are computed
    # with IEEE semantics like the reference's loops; the rest stay exact.
    rng = np.random.default_rng(11)
    M, K, N = 256, 128, 200
    a = rng.uniform(-1, 1, (M, K))
    b = rng.uniform(-1, 1, (K, N))
    a[3, 5] = np.nan
    a[100, 0] = np.inf
    b[7, 150] = -np.inf
    A = Pair(qs, a.ravel(order="F"), (M, K), (1, M))
    B = Pair(qs, b.ravel(order="F"), (K, N), (1, K))
    C = colmajor_pair(qs, rng, (M, N), "Float64")
    got, ref, plan = run_pair(qs, orc, C, 1.0, A, (1, 2), B, (2, 3), 0.5, (1, 3), method="ozaki",
                              precision=1)
    g = got.reshape(N, M).T
    r = ref.reshape(N, M).T
    assert np.array_equal(np.isnan(g), np.isnan(r))
    assert np.array_equal(np.isinf(g), np.isinf(r))
    fin = np.isfinite(r)
    assert np.all(g[fin] == g[fin])
    assert rel_fro(g[fin], r[fin]) <= TOL64


def test_ozaki_mixed_input_eltypes(qs, orc):
    # Float32 A with Float64 B and C: compute type Float64, conversion on load.
    rng = np.random.default_rng(12)
    A = uniform_pair(qs, rng, (300, 200), et="Float32")
    B = uniform_pair(qs, rng, (200, 260))
    C = colmajor_pair(qs, rng, (300, 260), "Float64")
    got, ref, plan = run_pair(qs, orc, C, 1.0, A, (1, 2), B, (2, 3), 1.0, (1, 3), precision=1, method="ozaki")
    assert plan.method == "ozaki"
    assert rel_fro(got, ref) <= TOL64


@pytest.mark.parametrize("MKN", [(256, 256, 256), (300, 200, 520), (1024, 512, 1024)])
def test_bf16x3_float32_matches_oracle(qs, orc, MKN):
    M, K, N = MKN
    rng = np.random.default_rng(M + N)
    A = uniform_pair(qs, rng, (M, K), et="Float32")
    B = uniform_pair(qs, rng, (K, N), et="Float32")
    C = colmajor_pair(qs, rng, (M, N), "Float32")
    plan = qs.plan_contract(C.dev, A.dev, (1, 2), B.dev, (2, 3), (1, 3), method="bf16x3")
    assert plan.method == "bf16x3"
    qs.execute(plan, 1.5, 0.5)
    got = C.device_parent()
    # FP64 oracle on the same Float32 inputs
    Ch = orc.HostView(C.host.parent.astype(np.float64), C.host.size, C.host.strides)
    Ah = orc.HostView(A.host.parent.astype(np.float64), A.host.size, A.host.strides)
    Bh = orc.HostView(B.host.parent.astype(np.float64), B.host.size, B.host.strides)
    orc.brute(Ch, 1.5, Ah, (1, 2), Bh, (2, 3), 0.5, (1, 3))
    assert rel_fro(got.astype(np.float64), Ch.parent) <= TOL32, rel_fro(got.astype(np.float64), Ch.parent)


def test_bf16x3_wide_exponents(qs, orc):
    rng = np.random.default_rng(13)
    A = uniform_pair(qs, rng, (256, 300), et="Float32", scale_axis=0)
    B = uniform_pair(qs, rng, (300, 384), et="Float32", scale_axis=1)
    C = colmajor_pair(qs, rng, (256, 384), "Float32", fill=np.nan)
    plan = qs.plan_contract(C.dev, A.dev, (1, 2), B.dev, (2, 3), (1, 3))
    qs.execute(plan, 1.0, 0.0)
    got = C.device_parent().astype(np.float64)
    Ch = orc.HostView(np.zeros(256 * 384), (256, 384), (1, 256))
    Ah = orc.HostView(A.host.parent.astype(np.float64), A.host.size, A.host.strides)
    Bh = orc.HostView(B.host.parent.astype(np.float64), B.host.size, B.host.strides)
    orc.brute(Ch, 1.0, Ah, (1, 2), Bh, (2, 3), 0.0, (1, 3))
    assert rel_fro(got, Ch.parent) <= TOL32


def complex_pair(qs, rng, shape, et="ComplexF64"):
    n = int(np.prod(shape))
    v = (rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n))
    v = v.astype(np.complex128 if et == "ComplexF64" else np.complex64)
    st, acc = [], 1
    for s in shape:
        st.append(acc)
        acc *= s
    return Pair(qs, v, tuple(shape), tuple(st))


@pytest.mark.parametrize("conj", [(False, False), (True, False), (False, True)])
@pytest.mark.parametrize("beta", [0.0, 0.5 - 0.25j])
def test_complex_1m_ozaki(qs, orc, conj, beta):
    # ComplexF64 through the 1m formulation: A as a 2M x 2K real "1e"
    # matrix, B as 2K x N "1r", on the INT8 Ozaki kernel.
    rng = np.random.default_rng(21)
    M, K, N = 200, 150, 260
    A = complex_pair(qs, rng, (M, K))
    B = complex_pair(qs, rng, (K, N))
    C = colmajor_pair(qs, rng, (M, N), "ComplexF64", fill=np.nan if beta == 0 else None)
    got, ref, plan = run_pair(qs, orc, C, 1.25 + 0.5j, A, (1, 2), B, (2, 3), beta, (1, 3),
                              conjA=conj[0], conjB=conj[1], precision=1, method="ozaki")
    assert plan.method == "ozaki" and plan.complex_mode == "1m"
    assert np.all(np.isfinite(got))
    assert rel_fro(got, ref) <= TOL64, rel_fro(got, ref)


@pytest.mark.parametrize("mode", ["planar", None])
@pytest.mark.parametrize("conj", [(False, False), (True, True), (False, True)])
@pytest.mark.parametrize("beta", [0.0, 0.5 - 0.25j])
def test_complex_planar_ozaki(qs, orc, mode, conj, beta):
    # The planar layout (A as [re | im] along K, B expanded to 2N interleaved
    # columns): C's Re/Im land in adjacent columns of one epilogue thread.
    # M > N, so the default picks it too.
    rng = np.random.default_rng(31)
    M, K, N = 300, 150, 140
    A = complex_pair(qs, rng, (M, K))
    B = complex_pair(qs, rng, (K, N))
    C = colmajor_pair(qs, rng, (M, N), "ComplexF64", fill=np.nan if beta == 0 else None)
    got, ref, plan = run_pair(qs, orc, C, 1.25 + 0.5j, A, (1, 2), B, (2, 3), beta, (1, 3),
                              conjA=conj[0], conjB=conj[1], precision=1, complex_mode=mode, method="ozaki")
    assert plan.method == "ozaki" and plan.complex_mode == "planar"
    assert np.all(np.isfinite(got))
    assert rel_fro(got, ref) <= TOL64, rel_fro(got, ref)


def test_complex_planar_nonfinite_and_f32(qs, orc):
    rng = np.random.default_rng(32)
    M, K, N = 260, 90, 140
    A = complex_pair(qs, rng, (M, K))
    b = (rng.standard_normal(K * N) + 1j * rng.standard_normal(K * N)) / np.sqrt(2)
    b[K * 7 + 3] = complex(np.inf, 0)  # column 7 of B
    B = Pair(qs, b, (K, N), (1, K))
    C = colmajor_pair(qs, rng, (M, N), "ComplexF64")
    got, ref, plan = run_pair(qs, orc, C, 1.0, A, (1, 2), B, (2, 3), 0.5, (1, 3), precision=1,
                              complex_mode="planar", method="ozaki")
    assert plan.complex_mode == "planar"
    g = got.reshape(N, M).T
    r = ref.reshape(N, M).T
    assert np.array_equal(np.isnan(g), np.isnan(r)) and np.array_equal(np.isinf(g), np.isinf(r))
    fin = np.isfinite(r)
    assert rel_fro(g[fin], r[fin]) <= TOL64
    # ComplexF32 through split BF16x3 in the planar layout
    A32 = complex_pair(qs, rng, (M, K), "ComplexF32")
    B32 = complex_pair(qs, rng, (K, N), "ComplexF32")
    C32 = colmajor_pair(qs, rng, (M, N), "ComplexF32")
    plan = qs.plan_contract(C32.dev, A32.dev, (1, 2), B32.dev, (2, 3), (1, 3), complex_mode="planar",
                            method="bf16x3")
    assert plan.method == "bf16x3" and plan.complex_mode == "planar"
    qs.execute(plan, 0.5 + 1j, 0.25)
    got = C32.device_parent().astype(np.complex128)
    Ch = orc.HostView(C32.host.parent.astype(np.complex128), C32.host.size, C32.host.strides)
    Ah = orc.HostView(A32.host.parent.astype(np.complex128), A32.host.size, A32.host.strides)
    Bh = orc.HostView(B32.host.parent.astype(np.complex128), B32.host.size, B32.host.strides)
    orc.brute(Ch, 0.5 + 1j, Ah, (1, 2), Bh, (2, 3), 0.25, (1, 3))
    assert rel_fro(got, Ch.parent) <= TOL32, rel_fro(got, Ch.parent)


def test_complex_mps_environment_steps(qs, orc):
    # The MPS environment update at chi = 64: T1 = L*A, T2 = T1*W,
    # out = T2*conj(A) (the last step conjugates on load).
    rng = np.random.default_rng(22)
    chi, D, d = 64, 5, 2
    L = complex_pair(qs, rng, (chi, D, chi))
    A = complex_pair(qs, rng, (chi, d, chi))
    W = complex_pair(qs, rng, (D, d, D, d))
    # labels: al=1, w=2, al'=3, s=4, be=5, w'=6, t=7, be'=8
    T1 = colmajor_pair(qs, rng, (D, chi, d, chi), "ComplexF64", fill=0)
    got, ref, p1 = run_pair(qs, orc, T1, 1, L, (1, 2, 3), A, (1, 4, 5), 0, (2, 3, 4, 5), precision=1,
                            method="ozaki")
    assert p1.method == "ozaki" and rel_fro(got, ref) <= TOL64
    T1.host.parent[:] = got  # continue from the device result on both sides
    T2 = colmajor_pair(qs, rng, (chi, chi, D, d), "ComplexF64", fill=0)
    got, ref, p2 = run_pair(qs, orc, T2, 1, T1, (2, 3, 4, 5), W, (2, 4, 6, 7), 0, (3, 5, 6, 7), precision=1)
    assert rel_fro(got, ref) <= TOL64
    T2.host.parent[:] = got
    O = colmajor_pair(qs, rng, (chi, D, chi), "ComplexF64", fill=0)
    got, ref, p3 = run_pair(qs, orc, O, 1, T2, (3, 5, 6, 7), A, (3, 7, 8), 0, (5, 6, 8), conjB=True,
                            precision=1)
    assert rel_fro(got, ref) <= TOL64  # N = chi = 64 < one tile: the gather kernel


def test_complex_times_real_and_nonfinite(qs, orc):
    rng = np.random.default_rng(23)
    M, K, N = 130, 90, 140
    A = complex_pair(qs, rng, (M, K))
    b = rng.uniform(-1, 1, K * N)
    b[5] = np.nan  # column 0 of B
    B = Pair(qs, b, (K, N), (1, K))
    C = colmajor_pair(qs, rng, (M, N), "ComplexF64")
    got, ref, plan = run_pair(qs, orc, C, 1.0, A, (1, 2), B, (2, 3), 1.0, (1, 3), precision=1, method="ozaki")
    assert plan.method == "ozaki"
    g = got.reshape(N, M).T
    r = ref.reshape(N, M).T
    assert np.array_equal(np.isnan(g), np.isnan(r))
    fin = np.isfinite(r)
    assert rel_fro(g[fin], r[fin]) <= TOL64


def test_complex_f32_bf16x3(qs, orc):
    rng = np.random.default_rng(24)
    M, K, N = 256, 200, 300
    A = complex_pair(qs, rng, (M, K), "ComplexF32")
    B = complex_pair(qs, rng, (K, N), "ComplexF32")
    C = colmajor_pair(qs, rng, (M, N), "ComplexF32")
    plan = qs.plan_contract(C.dev, A.dev, (1, 2), B.dev, (2, 3), (1, 3), conjA=True, method="bf16x3")
    assert plan.method == "bf16x3" and plan.complex_mode == "1m"
    qs.execute(plan, 0.5 + 1j, 0.25)
    got = C.device_parent().astype(np.complex128)
    Ch = orc.HostView(C.host.parent.astype(np.complex128), C.host.size, C.host.strides)
    Ah = orc.HostView(A.host.parent.astype(np.complex128), A.host.size, A.host.strides)
    Bh = orc.HostView(B.host.parent.astype(np.complex128), B.host.size, B.host.strides)
    orc.brute(Ch, 0.5 + 1j, Ah, (1, 2), Bh, (2, 3), 0.25, (1, 3), conjA=True)
    assert rel_fro(got, Ch.parent) <= TOL32, rel_fro(got, Ch.parent)
