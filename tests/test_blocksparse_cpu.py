"""Block-sparse front end, host side (no GPU): allowed blocks follow the
flux rule, block products pair equal charges of dual contracted legs (checked
against brute force), waves never put a C block twice, and leg errors."""
import importlib
import itertools

import pytest


@pytest.fixture(scope="module")
def bs(qs):
    return importlib.import_module(qs.__name__ + ".blocksparse")


def space(bs, qd, dual=False):
    return bs.U1Space(tuple(qd.items()), dual)


def test_allowed_keys_follow_the_flux_rule(bs):
    a = space(bs, {-1: 2, 0: 3, 1: 2})
    b = space(bs, {0: 4, 1: 1}, dual=True)
    keys = bs.allowed_keys([a, a, b], 1)
    want = [k for k in itertools.product(a.charges, a.charges, b.charges) if k[0] + k[1] - k[2] == 1]
    assert keys == want


def test_block_products_match_brute_force_and_waves_are_disjoint(bs):
    x = space(bs, {-1: 3, 0: 5, 1: 3})
    k1 = space(bs, {0: 4, 1: 2, 2: 1})
    k2 = space(bs, {-1: 2, 0: 2})
    y = space(bs, {0: 6, 1: 2})
    A_sp = [x, k1, k2]                     # A[a, k, l]
    B_sp = [k1.flip(), k2.flip(), y]       # B[k, l, b]
    Ak, Bk = bs.allowed_keys(A_sp, 0), bs.allowed_keys(B_sp, 1)
    prods, c_sp = bs.pair_blocks(A_sp, Ak, (1, 2, 3), B_sp, Bk, (2, 3, 4), (4, 1))
    assert c_sp == [y, x]
    brute = {(kb[2], ka[0], ka, kb) for ka in Ak for kb in Bk if ka[1] == kb[0] and ka[2] == kb[1]}
    assert {(p.kc[0], p.kc[1], p.ka, p.kb) for p in prods} == brute
    waves = bs.waves_of(prods)
    assert sum(len(w) for w in waves) == len(prods)
    for w in waves:
        assert len({p.kc for p in w}) == len(w)
    # every C key lies in the flux-1 sector of C
    assert {p.kc for p in prods} <= set(bs.allowed_keys(c_sp, 1))


def test_leg_errors(bs, qs):
    a = space(bs, {0: 2, 1: 2})
    with pytest.raises(qs.DimensionMismatch):       # contracted legs not dual
        bs.pair_blocks([a, a], [], (1, 2), [a, a], [], (2, 3), (1, 3))
    with pytest.raises(qs.DimensionMismatch):       # different sectors
        bs.pair_blocks([a, a], [], (1, 2), [space(bs, {0: 3, 1: 2}, True), a], [], (2, 3), (1, 3))
    with pytest.raises(qs.ArgumentError):
        bs.pair_blocks([a, a], [], (1, 2), [a.flip(), a], [], (2, 3), (1,))
    with pytest.raises(qs.ArgumentError):
        bs.U1Space(((0, 2), (0, 3)))
