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
