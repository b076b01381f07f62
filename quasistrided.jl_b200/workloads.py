"""Synthetic workloads of the engine's benchmark shapes (seeded).

u1_blocks: the uneven dense blocks of one U(1)-symmetric network step,
C[x,y,z] = sum_{k1,k2} A[x,k1,k2,y] * B[k2,z,k1], one independent contraction
per block.  Each leg's size is the dimension of a charge sector drawn
uniformly from 41 sectors q = -20..20 whose dimensions follow a discretised
Gaussian profile, dim(q) = clip(round(512 exp(-q^2 / (2 sigma^2))), 8, 512).
Per-block operand size is bounded: while |A| + |B| + |C| exceeds `cap`
elements the largest of A's legs (x, k1, k2, y) is halved (not below 8), so
the output leg z keeps its sector size.  Each block stores A and B with a
random axis order, so strides differ from block to block.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass

import numpy as np

SECTORS = 41


def sector_dims(sigma: float = 6.0) -> np.ndarray:
    q = np.arange(-(SECTORS // 2), SECTORS // 2 + 1)
    return np.clip(np.round(512 * np.exp(-q.astype(np.float64) ** 2 / (2 * sigma * sigma))), 8, 512).astype(np.int64)


@dataclass
class Block:
    x: int
    k1: int
    k2: int
    y: int
    z: int
    permA: tuple  # storage order of A's logical axes (x, k1, k2, y)
    permB: tuple  # storage order of B's logical axes (k2, z, k1)

    @property
    def flops(self) -> int:
        return 2 * self.x * self.y * self.z * self.k1 * self.k2

    @property
    def elems(self) -> tuple:
        a = self.x * self.k1 * self.k2 * self.y
        b = self.k2 * self.z * self.k1
        c = self.x * self.y * self.z
        return a, b, c

    # Labels: x=1, y=2, z=3, k1=-1, k2=-2 (TensorOperations' convention).
    def a_shape_labels(self):
        dims = (self.x, self.k1, self.k2, self.y)
        labs = (1, -1, -2, 2)
        return tuple(dims[i] for i in self.permA), tuple(labs[i] for i in self.permA)

    def b_shape_labels(self):
        dims = (self.k2, self.z, self.k1)
        labs = (-2, 3, -1)
        return tuple(dims[i] for i in self.permB), tuple(labs[i] for i in self.permB)

    def c_shape_labels(self):
        return (self.x, self.y, self.z), (1, 2, 3)


def u1_blocks(n: int = 2000, seed: int = 0, cap: int = 1 << 21, sigma: float = 6.0) -> list:
    rng = np.random.default_rng(seed)
    dims = sector_dims(sigma)
    permsA = list(itertools.permutations(range(4)))
    permsB = list(itertools.permutations(range(3)))
    out = []
    for _ in range(n):
        legs = dims[rng.integers(0, SECTORS, 5)].astype(np.int64)  # x, k1, k2, y, z

        def total(l):
            x, k1, k2, y, z = (int(v) for v in l)
            return x * k1 * k2 * y + k2 * z * k1 + x * y * z

        while total(legs) > cap:
            i = int(np.argmax(legs[:4])) if legs[:4].max() > 8 else 4
            if legs[i] <= 8:
                break
            legs[i] = max(8, legs[i] // 2)
        pa = permsA[rng.integers(0, len(permsA))]
        pb = permsB[rng.integers(0, len(permsB))]
        x, k1, k2, y, z = (int(v) for v in legs)
        out.append(Block(x, k1, k2, y, z, tuple(pa), tuple(pb)))
    return out


def histogram(blocks, edges=(8, 16, 32, 64, 128, 256, 512, 1024, 4096, 1 << 14, 1 << 16, 1 << 18, 1 << 20)):
    """Realised sizes: counts of M = x*y, N = z and K = k1*k2 per bin
    [edges[i], edges[i+1]), plus totals."""
    M = np.array([b.x * b.y for b in blocks])
    N = np.array([b.z for b in blocks])
    K = np.array([b.k1 * b.k2 for b in blocks])
    e = np.array(list(edges) + [np.iinfo(np.int64).max])
    h = lambda v: np.histogram(v, bins=e)[0].tolist()  # noqa: E731
    el = np.array([sum(b.elems) for b in blocks], dtype=np.float64)
    return {
        "edges": list(edges),
        "M": h(M), "N": h(N), "K": h(K),
        "blocks": len(blocks),
        "flops": float(sum(b.flops for b in blocks)),
        "elements": float(el.sum()),
        "max_block_elements": float(el.max()) if len(el) else 0.0,
    }


# ------------------------------------------------------------- serving ---
# A stream of contraction requests: Poisson arrivals at `rate` per second;
# shapes drawn uniformly from the permuted-matmul (96x128x32 . 128x80), the
# permuted 4-index contraction (a..d = 64, e = f = 48), the three pairwise
# steps of an MPS environment update (chi = 1024, D_W = 5, d = 2), one
# uneven U(1) block, and random rank-2..6 operand pairs (1e3..1e8 elements in
# total, log-uniform, 1-3 contracted labels, random label order); eltypes
# Float32 / Float64 / ComplexF64 in 40/40/20 proportion; 30% of the requests
# use a device-resident operand (one per shape family and eltype) as A.

SERVING_DTYPES = (np.float32, np.float64, np.complex128)
SERVING_DTYPE_P = (0.4, 0.4, 0.2)


def _family_shapes(fam, rng):
    """(shapeA, indA, shapeB, indB, indC) of one request of family `fam`."""
    if fam == "matmul":
        return (96, 128, 32), (1, 2, 3), (128, 80), (2, 4), (1, 4, 3)
    if fam == "permuted4":
        return (64, 48, 64, 48), (1, 5, 2, 6), (48, 64, 48, 64), (6, 3, 5, 4), (1, 2, 3, 4)
    if fam == "mps1":   # T1[w,al',s,be] = L[al,w,al'] * A[al,s,be]
        return (1024, 5, 1024), (1, 2, 3), (1024, 2, 1024), (1, 4, 5), (2, 3, 4, 5)
    if fam == "mps2":   # T2[al',be,w',t] = T1[w,al',s,be] * W[w,s,w',t]
        return (5, 1024, 2, 1024), (1, 2, 3, 4), (5, 2, 5, 2), (1, 3, 5, 6), (2, 4, 5, 6)
    if fam == "mps3":   # out[be,w',be'] = T2[al',be,w',t] * A[al',t,be']
        return (1024, 1024, 5, 2), (1, 2, 3, 4), (1024, 2, 1024), (1, 4, 5), (2, 3, 5)
    if fam == "block":
        b = u1_blocks(n=1, seed=int(rng.integers(1 << 30)))[0]
        sa, la = b.a_shape_labels()
        sb, lb = b.b_shape_labels()
        sc, lc = b.c_shape_labels()
        return sa, la, sb, lb, lc
    # random pair
    k = int(rng.integers(1, 4))
    fa = int(rng.integers(max(1, 2 - k), 6 - k + 1))
    fb = int(rng.integers(max(1, 2 - k), 6 - k + 1))
    total = 10 ** rng.uniform(3, 8)
    nlab = fa + fb + k
    # leg sizes: log-uniform around total^(1/rank of the largest operand)
    r = max(fa + k, fb + k)
    base = max(2.0, total ** (1.0 / r) / 1.5)
    sizes = [max(1, int(base * 2 ** rng.uniform(-1, 1))) for _ in range(nlab)]

    def nel(sz):
        a = np.prod([sizes[i] for i in range(fa)] + [sizes[fa + fb + j] for j in range(k)])
        bb = np.prod([sizes[fa + i] for i in range(fb)] + [sizes[fa + fb + j] for j in range(k)])
        c = np.prod([sizes[i] for i in range(fa + fb)])
        return a + bb + c

    while nel(sizes) > 1e8:
        j = int(np.argmax(sizes))
        sizes[j] = max(1, sizes[j] // 2)
    labs = list(range(1, nlab + 1))
    freeA, freeB, con = labs[:fa], labs[fa:fa + fb], labs[fa + fb:]
    la = freeA + con
    lb = con + freeB
    rng.shuffle(la)
    rng.shuffle(lb)
    lc = freeA + freeB
    rng.shuffle(lc)
    size_of = {l: sizes[l - 1] for l in labs}
    return (tuple(size_of[l] for l in la), tuple(la), tuple(size_of[l] for l in lb), tuple(lb), tuple(lc))


FAMILIES = ("matmul", "permuted4", "mps1", "mps2", "mps3", "block", "random")


def serving_stream(n: int, rate: float, seed: int = 0, reuse: float = 0.3, pool_elems: int = 1 << 26):
    """n requests with Poisson arrival offsets (seconds) at `rate` per second.

    Returns (specs, offsets, residents): specs are dicts with shapes, labels,
    dtype, alpha/beta and, for reuse, the resident key of A; residents maps
    key -> (shape, dtype).  Families are drawn uniformly; the three MPS steps
    count as one family.  No operand (C included) may exceed `pool_elems`
    elements: the
    values are column-major views into per-dtype pools (`pool_arrays`,
    `colmajor_view`), so a stream of large requests needs no per-request
    host copies.
    """
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, n)
    offsets = np.cumsum(gaps) - gaps[0]
    fams = ("matmul", "permuted4", "mps", "block", "random")
    specs, residents = [], {}
    for i in range(n):
        # A reusing request takes its A from the resident operand of a fixed
        # family (one per family and eltype); the others draw any family.
        reusing = rng.uniform() < reuse
        pick = fams[:3] if reusing else fams
        fam = pick[int(rng.integers(len(pick)))]
        if fam == "mps":
            fam = ("mps1", "mps2", "mps3")[int(rng.integers(3))]
        dt = SERVING_DTYPES[int(rng.choice(3, p=SERVING_DTYPE_P))]
        sa, la, sb, lb, lc = _family_shapes(fam, rng)

        def c_elems():
            d = dict(zip(la, sa))
            d.update(zip(lb, sb))
            return int(np.prod([d[l] for l in lc])) if lc else 1

        while max(int(np.prod(sa)), int(np.prod(sb)), c_elems()) > pool_elems:
            fam = "random"
            sa, la, sb, lb, lc = _family_shapes(fam, rng)
        res_key = None
        if reusing and fam != "random":
            res_key = f"{fam}:{np.dtype(dt).name}"
            residents.setdefault(res_key, (sa, dt))
        beta = 0.0 if rng.uniform() < 0.5 else 0.5
        specs.append({"family": fam, "shapeA": sa, "indA": la, "shapeB": sb, "indB": lb, "indC": lc,
                      "dtype": dt, "alpha": 1.0, "beta": beta, "resident": res_key})
    return specs, offsets, residents


def pool_arrays(pool_elems: int, seed: int = 1, dtypes=SERVING_DTYPES, allocate=None):
    """Seeded N(0,1) value pools, one per dtype.  `allocate(n, dtype)` may
    supply the storage (e.g. pinned host memory)."""
    rng = np.random.default_rng(seed)
    out = {}
    for dt in dtypes:
        buf = allocate(pool_elems, dt) if allocate else np.empty(pool_elems, dtype=dt)
        if np.issubdtype(np.dtype(dt), np.complexfloating):
            buf.real[:] = rng.standard_normal(pool_elems)
            buf.imag[:] = rng.standard_normal(pool_elems)
            buf /= np.sqrt(2.0)
        else:
            buf[:] = rng.standard_normal(pool_elems)
        out[np.dtype(dt)] = buf
    return out


def colmajor_view(pool_buf, shape, start: int = 0):
    n = int(np.prod(shape)) if len(shape) else 1
    return pool_buf[start:start + n].reshape(shape, order="F")
