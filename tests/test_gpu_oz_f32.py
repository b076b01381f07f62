"""Single precision through the Ozaki INT8 path (4 digits, 10 slice products,
the default tensor-core method for Float32/ComplexF32): against the FP64
oracle on the same Float32 values (alpha/beta rounded to Float32 first),
within 1e-6 (about the final rounding to Float32; split BF16x3 keeps ~1e-5),
for uniform and wide-exponent inputs, complex with conj, and the CTA-pair
kernel bitwise equal to the one-SM kernel at 4 slices."""
import numpy as np
import pytest
import torch

from _util import Pair, colmajor_pair, randn, rel_fro

pytestmark = pytest.mark.gpu


def oracle_f64(orc, C, alpha, A, indA, B, indB, beta, indC, **kw):
    f = lambda v: orc.HostView(v.parent.astype(np.complex128 if np.iscomplexobj(v.parent) else np.float64),  # noqa
                               v.size, v.strides, v.offset, v.op)
    Ch = f(C.host)
    orc.brute(Ch, alpha, f(A.host), indA, f(B.host), indB, beta, indC, **kw)
    return Ch.parent


@pytest.mark.parametrize("wide", [False, True])
def test_float32_auto_is_ozaki4(qs, orc, wide):
    rng = np.random.default_rng(41 + wide)
    M, K, N = 512, 600, 384
    A = colmajor_pair(qs, rng, (M, K), "Float32")
    B = colmajor_pair(qs, rng, (K, N), "Float32")
    if wide:
        for P, shape, axis in ((A, (M, K), 0), (B, (K, N), 1)):
            sc = np.exp2(rng.integers(-20, 21, shape[axis])).astype(np.float32)
            arr = P.host.parent.reshape(shape, order="F") * (sc[:, None] if axis == 0 else sc[None, :])
            P.host.parent[:] = arr.ravel(order="F")
            P.dev.parent.copy_(torch.from_numpy(P.host.parent))
    C = colmajor_pair(qs, rng, (M, N), "Float32")
    plan = qs.plan_contract(C.dev, A.dev, (1, 2), B.dev, (2, 3), (1, 3))
    assert plan.method == "ozaki" and plan.ozaki_slices == 4
    alpha, beta = 1.3, 0.7
    qs.execute(plan, alpha, beta)
    torch.cuda.synchronize()
    ref = oracle_f64(orc, C, float(np.float32(alpha)), A, (1, 2), B, (2, 3), float(np.float32(beta)), (1, 3))
    assert rel_fro(C.device_parent().astype(np.float64), ref) <= 1e-6


def test_complex_float32_ozaki_conj(qs, orc):
    rng = np.random.default_rng(43)
    M, K, N = 320, 260, 256
    A = colmajor_pair(qs, rng, (M, K), "ComplexF32")
    B = colmajor_pair(qs, rng, (K, N), "ComplexF32")
    C = colmajor_pair(qs, rng, (M, N), "ComplexF32")
    plan = qs.plan_contract(C.dev, A.dev, (1, 2), B.dev, (2, 3), (1, 3), conjB=True, method="ozaki")
    assert plan.ozaki_slices == 4
    qs.execute(plan, 0.5 - 1j, 0.25)
    torch.cuda.synchronize()
    ref = oracle_f64(orc, C, 0.5 - 1j, A, (1, 2), B, (2, 3), 0.25, (1, 3), conjB=True)
    assert rel_fro(C.device_parent().astype(np.complex128), ref) <= 1e-6


def test_pair_kernel_bitwise_at_four_slices(qs):
    rng = np.random.default_rng(44)
    M, K, N = 640, 512, 300                  # 5 M tiles: an odd pair
    A = colmajor_pair(qs, rng, (M, K), "Float32")
    B = colmajor_pair(qs, rng, (K, N), "Float32")
    c0 = randn(rng, M * N, "Float32")
    C0, C1 = Pair(qs, c0, (M, N), (1, M)), Pair(qs, c0, (M, N), (1, M))
    p1 = qs.plan_contract(C0.dev, A.dev, (1, 2), B.dev, (2, 3), (1, 3), method="ozaki", oz_single_sm=True)
    p2 = qs.plan_contract(C1.dev, A.dev, (1, 2), B.dev, (2, 3), (1, 3), method="ozaki")
    qs.execute(p1, 1.0, 0.5)
    qs.execute(p2, 1.0, 0.5)
    torch.cuda.synchronize()
    assert np.array_equal(C0.device_parent(), C1.device_parent())
