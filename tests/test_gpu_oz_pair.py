"""The CTA-pair Ozaki GEMM (tcgen05 cta_group::2, the default for 6 and 7
slices) against the one-SM kernel: the INT32 slice sums are exact and the
FP64 epilogue is the same, so C must be bitwise identical.  Even and odd
numbers of M tiles (the odd pair's second CTA computes padding rows that are
never stored), ragged N, beta != 0, strided C, both complex layouts, 7 slices;
and the result against the FP64 oracle."""
import numpy as np
import pytest
import torch

from _util import Pair, colmajor_pair, randn, rel_fro

pytestmark = pytest.mark.gpu


def both(qs, C0, C1, A, indA, B, indB, indC, alpha, beta, **kw):
    p1 = qs.plan_contract(C0.dev, A.dev, indA, B.dev, indB, indC, method="ozaki", oz_single_sm=True, **kw)
    p2 = qs.plan_contract(C1.dev, A.dev, indA, B.dev, indB, indC, method="ozaki", **kw)
    qs.execute(p1, alpha, beta)
    qs.execute(p2, alpha, beta)
    torch.cuda.synchronize()
    qs.check_status(p2)
    return p1, p2


@pytest.mark.parametrize("MKN", [(1024, 1152, 1024), (640, 512, 384), (130, 300, 100), (128, 256, 600),
                                 (2000, 700, 260)])
def test_pair_kernel_bitwise_equal_to_single_sm(qs, orc, MKN):
    M, K, N = MKN
    rng = np.random.default_rng(M + 3 * K + 7 * N)
    A = colmajor_pair(qs, rng, (M, K), "Float64")
    B = colmajor_pair(qs, rng, (K, N), "Float64")
    c0 = randn(rng, M * N, "Float64")
    C0 = Pair(qs, c0, (M, N), (1, M))
    C1 = Pair(qs, c0, (M, N), (1, M))
    p1, p2 = both(qs, C0, C1, A, (1, 2), B, (2, 3), (1, 3), 1.25, 0.5)
    assert p2.ozaki_slices == p1.ozaki_slices
    assert np.array_equal(C0.device_parent(), C1.device_parent())
    orc.brute(C1.host, 1.25, A.host, (1, 2), B.host, (2, 3), 0.5, (1, 3), precision=1)
    assert rel_fro(C1.device_parent(), C1.host.parent) <= 1e-13


@pytest.mark.parametrize("mode", ["planar", "1m"])
def test_pair_kernel_complex_and_strided(qs, mode):
    rng = np.random.default_rng(5)
    M, K, N = 300, 260, 200
    A = colmajor_pair(qs, rng, (M, K), "ComplexF64")
    B = colmajor_pair(qs, rng, (K, N), "ComplexF64")
    par = randn(rng, 3 * M * N + 50, "ComplexF64")
    C0 = Pair(qs, par, (M, N), (2, 2 * M + 1), 11)     # strided window of C
    C1 = Pair(qs, par, (M, N), (2, 2 * M + 1), 11)
    p1, p2 = both(qs, C0, C1, A, (1, 2), B, (2, 3), (1, 3), 0.5 - 1j, 2.0, complex_mode=mode)
    assert p2.complex_mode == mode and p2.ozaki_slices == 7
    assert np.array_equal(C0.device_parent(), C1.device_parent())


def test_pair_kernel_seven_slices_long_k(qs):
    rng = np.random.default_rng(9)
    M, K, N = 512, 4608, 256     # K > 4096: 7 slices
    A = colmajor_pair(qs, rng, (M, K), "Float64")
    B = colmajor_pair(qs, rng, (K, N), "Float64")
    C0 = colmajor_pair(qs, rng, (M, N), "Float64", fill=np.nan)
    C1 = colmajor_pair(qs, rng, (M, N), "Float64", fill=np.nan)
    p1, p2 = both(qs, C0, C1, A, (1, 2), B, (2, 3), (1, 3), 1.0, 0.0)
    assert p2.ozaki_slices == 7
    assert np.array_equal(C0.device_parent(), C1.device_parent())
