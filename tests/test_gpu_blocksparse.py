"""Block-sparse U(1) contractions on the device (grouped problem tables in
waves) against the dense contraction of the same tensors: real and complex
with conj, beta on existing C including blocks no product reaches,
persistent vs sequential groups, and reuse of a planned contraction."""
import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def bs(qs):
    return importlib.import_module(qs.__name__ + ".blocksparse")


def sp(bs, qd, dual=False):
    return bs.U1Space(tuple(qd.items()), dual)


def legs(bs):
    x = sp(bs, {-2: 9, -1: 17, 0: 33, 1: 17, 2: 9, 7: 5})   # charge 7 is never balanced
    k1 = sp(bs, {-1: 12, 0: 40, 1: 12})
    k2 = sp(bs, {0: 20, 1: 6})
    y = sp(bs, {-1: 30, 0: 64, 1: 30, 2: 8})
    return x, k1, k2, y


@pytest.mark.parametrize("dtype", [torch.float64, torch.complex128])
def test_block_contraction_matches_dense(qs, bs, dtype):
    x, k1, k2, y = legs(bs)
    A = bs.BlockSparseTensor.random([x, k1, k2], 0, dtype, seed=1)            # A[a,k,l]
    B = bs.BlockSparseTensor.random([k2.flip(), y, k1.flip()], 1, dtype, seed=2)  # B[l,b,k]
    conj = dtype.is_complex
    C = bs.contract(A, (1, 2, 3), B, (3, 4, 2), (4, 1), conjB=conj)            # C[b,a]
    assert C.flux == 1
    Ad, Bd = A.to_dense(), B.to_dense()
    want = np.einsum("akl,lbk->ba", Ad, np.conj(Bd) if conj else Bd)
    got = C.to_dense()
    assert np.linalg.norm(got - want) <= 1e-13 * np.linalg.norm(want)


def test_beta_on_existing_c_and_untouched_blocks(qs, bs):
    x, k1, k2, y = legs(bs)
    A = bs.BlockSparseTensor.random([x, k1, k2], 0, seed=3)
    B = bs.BlockSparseTensor.random([k2.flip(), y, k1.flip()], 1, seed=4)
    C = bs.BlockSparseTensor.random([y, x], 1, seed=5)
    c0 = C.to_dense()
    bc = bs.BlockContraction(C, A, (1, 2, 3), B, (3, 4, 2), (4, 1))
    assert bc.untouched and len(bc.waves) > 1       # charge-7 rows get no product; several waves
    bc.execute(1.5, 0.5)
    torch.cuda.synchronize()
    want = 1.5 * np.einsum("akl,lbk->ba", A.to_dense(), B.to_dense()) + 0.5 * c0
    assert np.linalg.norm(C.to_dense() - want) <= 1e-13 * np.linalg.norm(want)
    # reuse with another alpha, beta = 0 (C's old values never read)
    C.buffer.fill_(float("nan"))
    bc.execute(-2.0, 0.0)
    torch.cuda.synchronize()
    want = -2.0 * np.einsum("akl,lbk->ba", A.to_dense(), B.to_dense())
    got = C.to_dense()
    assert np.all(np.isfinite(got)) and np.linalg.norm(got - want) <= 1e-13 * np.linalg.norm(want)
    bc.release()


def test_sequential_groups_equal_persistent(qs, bs):
    x, k1, k2, y = legs(bs)
    A = bs.BlockSparseTensor.random([x, k1, k2], 0, torch.float32, seed=6)
    B = bs.BlockSparseTensor.random([k2.flip(), y, k1.flip()], 1, torch.float32, seed=7)
    C1 = bs.contract(A, (1, 2, 3), B, (3, 4, 2), (4, 1), mode="persistent")
    C2 = bs.contract(A, (1, 2, 3), B, (3, 4, 2), (4, 1), mode="sequential")
    assert torch.equal(C1.buffer, C2.buffer)
