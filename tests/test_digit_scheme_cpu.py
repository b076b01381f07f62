"""The Ozaki digit scheme of the pack, modelled on the CPU.

Each row is scaled by 2^-E (E = frexp exponent of its max |x|, + 1) and by
127/128, rounded once to the integer q = x * 127/128 * 2^(8s-E), and the s
bytes of q + sum_i 128 * 256^i, minus 128, are its balanced base-256 digits
(leading digit first).  The GEMM keeps the slice products with p + q <= s - 1
(0-based), accumulates each diagonal exactly in integers and weights it by
(128/127)^2 * 256^-(p+q+2).  These tests check, in exact or FP64
arithmetic, that every digit is an exact int8, that the digits reconstruct
the row within one rounding of q, that the single-FMA rounding the kernel
uses for s <= 6 (adding 1.5 * 2^52 and reading the low bits) equals
round-to-nearest, and that a truncated dot product lands within the stated
error of the exact one.
"""
import struct

import numpy as np
import pytest

MAGIC = 6755399441055744.0  # 1.5 * 2^52


def row_digits(row, s):
    mb = np.max(np.abs(row))
    _, e = np.frexp(mb)
    E = int(e) + 1
    f = 127.0 / 128.0 * 2.0 ** (8 * s - E)
    q = np.rint(row * f).astype(np.int64)
    bias = 0x8080808080808080 >> (64 - 8 * s)
    u = (q + bias).astype(np.uint64)
    planes = []
    for p in range(s):
        b = (u >> np.uint64(8 * (s - 1 - p))) & np.uint64(0xFF)
        planes.append(b.astype(np.int64) - 128)
    return E, q, bias, np.array(planes)


def reconstruct(E, planes):
    s = planes.shape[0]
    acc = sum(planes[p].astype(np.float64) * 256.0 ** -(p + 1) for p in range(s))
    return acc * 2.0 ** E * 128.0 / 127.0


@pytest.mark.parametrize("s", [4, 6, 7])
def test_digits_are_int8_and_reconstruct(s):
    rng = np.random.default_rng(s)
    for trial in range(300):
        row = rng.uniform(-1, 1, 97) * 2.0 ** int(rng.integers(-60, 60))
        if trial % 3 == 0:
            row *= 2.0 ** rng.uniform(-25, 25, row.size)  # wide exponents inside the row
        E, q, bias, P = row_digits(row, s)
        assert np.all(q + bias >= 0) and np.all(q + bias < 2 ** (8 * s))
        assert P.min() >= -128 and P.max() <= 127
        assert np.abs(P[0]).max() <= 127  # the leading digit
        err = np.max(np.abs(reconstruct(E, P) - row))
        # one rounding of q: 2^-(8s+1) * 128/127 * 2^E, plus FP64 slack for s = 7
        bound = 2.0 ** (-(8 * s + 1)) * 128.0 / 127.0 * 2.0 ** E * (1 + 1e-9)
        bound += 4 * np.finfo(np.float64).eps * np.max(np.abs(row))
        assert err <= bound, (s, trial, err, bound)


@pytest.mark.parametrize("s", [4, 6])
def test_single_fma_rounding_matches_rint(s):
    # bits(v*f + 1.5*2^52) + (bias - 2^51), low 8s bits, is q + bias
    rng = np.random.default_rng(100 + s)
    bias = 0x8080808080808080 >> (64 - 8 * s)
    for _ in range(3000):
        v = rng.uniform(-1, 1) * 2.0 ** int(rng.integers(-40, 40))
        _, e = np.frexp(abs(v) * rng.uniform(1, 3))
        f = 127.0 / 128.0 * 2.0 ** (8 * s - (int(e) + 1))
        # the kernel adds MAGIC to the exact product in one FMA; numpy rounds
        # the product first, which leaves the bit extraction under test the same
        y = v * f
        t = y + MAGIC
        bits = struct.unpack("<Q", struct.pack("<d", t))[0]
        got = (bits + bias - (1 << 51)) & ((1 << (8 * s)) - 1)
        assert got == int(np.rint(y)) + bias


@pytest.mark.parametrize("s", [4, 6, 7])
def test_truncated_dot_product(s):
    rng = np.random.default_rng(7 + s)
    K = 2304
    a = rng.uniform(-1, 1, K)
    b = rng.uniform(-1, 1, K) * 2.0 ** 17
    Ea, _, _, Pa = row_digits(a, s)
    Eb, _, _, Pb = row_digits(b, s)
    acc = 0.0
    for t in range(s):  # diagonals kept: p + q = t, t <= s - 1
        diag = sum(int(np.dot(Pa[p], Pb[t - p])) for p in range(t + 1))  # exact integers
        acc += diag * (128.0 / 127.0) ** 2 * 256.0 ** -(t + 2)
    acc *= 2.0 ** (Ea + Eb)
    exact = float(np.dot(a.astype(np.longdouble), b.astype(np.longdouble)))
    scale = np.linalg.norm(a) * np.linalg.norm(b)
    # dropped diagonals and the rounding of q: a few 256^-s of the scale
    assert abs(acc - exact) / scale <= 8 * 256.0 ** -s + 1e-15
