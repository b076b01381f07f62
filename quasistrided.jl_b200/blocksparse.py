"""Block-sparse (U(1)-symmetric) tensors on the device, contracted through
grouped problem tables.

The reference contracts one strided array pair per call; symmetric tensor
networks (TensorKit-style U(1) sectors) turn one contraction into many
independent block products of uneven sizes.  This front end emits them as
the grouped engine's problem tables (``ContractGroup``, persistent mode: one
launch per stage and kernel class for all blocks):

* every leg is a ``U1Space``: charge -> sector dimension, and a duality;
* a tensor stores only the blocks whose charges add up to its flux
  (sum over legs of +q, or -q on dual legs), all in one device buffer,
  each block a column-major view;
* contracted legs must be dual to each other with equal sectors; a C block
  receives one product per matching charge of the contracted legs.  Products
  into the same C block are put in different *waves* (wave w holds the w-th
  product of every C block), so one grouped launch never writes a C block
  twice; the first product of a block applies beta, later ones beta = 1.
  C blocks no product reaches are scaled by beta with the device add kernel.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _abi

Key = Tuple[int, ...]


@dataclass(frozen=True)
class U1Space:
    """A leg: ``sectors`` = ((charge, dimension), ...), charges distinct;
    ``dual`` flips the sign the charges carry in the flux rule."""

    sectors: Tuple[Tuple[int, int], ...]
    dual: bool = False

    def __post_init__(self):
        qs = [q for q, _ in self.sectors]
        if len(set(qs)) != len(qs) or any(d < 0 for _, d in self.sectors):
            raise _abi.ArgumentError("U1Space: charges must be distinct and dimensions >= 0")
        object.__setattr__(self, "sectors", tuple(sorted((int(q), int(d)) for q, d in self.sectors)))

    @property
    def charges(self) -> Tuple[int, ...]:
        return tuple(q for q, _ in self.sectors)

    def dim(self, q: int) -> int:
        for c, d in self.sectors:
            if c == q:
                return d
        return 0

    @property
    def total(self) -> int:
        return sum(d for _, d in self.sectors)

    def offset(self, q: int) -> int:
        """Start of sector q in the dense (charge-ordered) leg."""
        o = 0
        for c, d in self.sectors:
            if c == q:
                return o
            o += d
        raise KeyError(q)

    def flip(self) -> "U1Space":
        return U1Space(self.sectors, not self.dual)

    @property
    def sign(self) -> int:
        return -1 if self.dual else 1


def allowed_keys(spaces: Sequence[U1Space], flux: int) -> List[Key]:
    """Charge tuples (one per leg) of the blocks a tensor of this flux holds."""
    out = []
    for key in itertools.product(*[s.charges for s in spaces]):
        if sum(s.sign * q for s, q in zip(spaces, key)) == flux and \
                all(s.dim(q) > 0 for s, q in zip(spaces, key)):
            out.append(tuple(key))
    return out


class BlockSparseTensor:
    """Blocks of a U(1)-symmetric tensor in one device buffer (column-major
    blocks, charge order of the keys)."""

    def __init__(self, spaces: Sequence[U1Space], flux: int = 0, dtype=torch.float64, device="cuda",
                 fill: Optional[float] = 0.0, buffer: Optional[torch.Tensor] = None):
        self.spaces = tuple(spaces)
        self.flux = int(flux)
        self.dtype = dtype
        self.keys = allowed_keys(self.spaces, self.flux)
        self.offsets: Dict[Key, int] = {}
        n = 0
        for k in self.keys:
            self.offsets[k] = n
            n += int(np.prod(self.block_shape(k)))
        self.size = n
        if buffer is not None:
            if buffer.numel() < max(n, 1) or buffer.dtype != dtype:
                raise _abi.ArgumentError("BlockSparseTensor: buffer too small or of another dtype")
            self.buffer = buffer
        elif fill is None:
            self.buffer = torch.empty(max(n, 1), dtype=dtype, device=device)
        else:
            self.buffer = torch.full((max(n, 1),), fill, dtype=dtype, device=device)

    def block_shape(self, key: Key) -> Tuple[int, ...]:
        return tuple(s.dim(q) for s, q in zip(self.spaces, key))

    def block(self, key: Key):
        """The block as a column-major StridedView into the buffer."""
        from . import StridedView
        shape = self.block_shape(key)
        strides, acc = [], 1
        for d in shape:
            strides.append(acc)
            acc *= d
        return StridedView(self.buffer, shape, tuple(strides), self.offsets[key])

    @classmethod
    def random(cls, spaces, flux=0, dtype=torch.float64, seed=0, device="cuda") -> "BlockSparseTensor":
        t = cls(spaces, flux, dtype, device, fill=None)
        g = torch.Generator(device=device).manual_seed(seed)
        t.buffer.copy_(torch.randn(t.buffer.numel(), dtype=dtype, device=device, generator=g))
        return t

    def to_dense(self) -> np.ndarray:
        """The dense array (zeros outside the blocks) on the host."""
        buf = self.buffer.detach().cpu().numpy()
        out = np.zeros(tuple(s.total for s in self.spaces), dtype=buf.dtype)
        for k in self.keys:
            shape = self.block_shape(k)
            n = int(np.prod(shape))
            blk = buf[self.offsets[k]:self.offsets[k] + n].reshape(shape, order="F")
            sl = tuple(slice(s.offset(q), s.offset(q) + d) for s, q, d in zip(self.spaces, k, shape))
            out[sl] = blk
        return out


@dataclass
class BlockProduct:
    """One block product: C[kc] (+)= A[ka] * B[kb]."""
    kc: Key
    ka: Key
    kb: Key


def pair_blocks(A_spaces, A_keys, indA, B_spaces, B_keys, indB, indC) -> Tuple[List[BlockProduct], List[U1Space]]:
    """Block products of C[indC] = A[indA] * B[indB] and the spaces of C's
    legs, after checking the legs: contracted legs dual with equal sectors,
    free legs passed through to C."""
    indA, indB, indC = tuple(indA), tuple(indB), tuple(indC)
    if len(indA) != len(A_spaces) or len(indB) != len(B_spaces):
        raise _abi.ArgumentError("pair_blocks: one label per leg")
    cl = [l for l in indA if l in indB]
    for l in cl:
        if l in indC:
            raise _abi.ArgumentError(f"label {l} is in A, B and C")
        sa, sb = A_spaces[indA.index(l)], B_spaces[indB.index(l)]
        if sa.sectors != sb.sectors or sa.dual == sb.dual:
            raise _abi.DimensionMismatch(f"contracted label {l}: the legs must be dual with equal sectors")
    c_spaces = []
    for l in indC:
        if l in indA and l not in indB:
            c_spaces.append(A_spaces[indA.index(l)])
        elif l in indB and l not in indA:
            c_spaces.append(B_spaces[indB.index(l)])
        else:
            raise _abi.ArgumentError(f"label {l} of indC must be a free label of exactly one of A, B")
    if sorted(l for l in indA + indB if l not in cl) != sorted(indC):
        raise _abi.ArgumentError("every free label of A and B must appear in indC once")
    ia = [indA.index(l) for l in cl]
    ib = [indB.index(l) for l in cl]
    by_charge: Dict[Key, List[Key]] = {}
    for ka in A_keys:
        by_charge.setdefault(tuple(ka[i] for i in ia), []).append(ka)
    prods = []
    for kb in B_keys:
        for ka in by_charge.get(tuple(kb[i] for i in ib), ()):
            kc = tuple(ka[indA.index(l)] if l in indA else kb[indB.index(l)] for l in indC)
            prods.append(BlockProduct(kc, ka, kb))
    return prods, c_spaces


def waves_of(products: Sequence[BlockProduct]) -> List[List[BlockProduct]]:
    """Wave w = the w-th product of every C block (C blocks distinct per wave)."""
    per: Dict[Key, List[BlockProduct]] = {}
    for p in products:
        per.setdefault(p.kc, []).append(p)
    nw = max((len(v) for v in per.values()), default=0)
    return [[v[w] for v in per.values() if len(v) > w] for w in range(nw)]


class BlockContraction:
    """``C = alpha * contract(A[indA], B[indB]) + beta * C`` over all blocks,
    planned once: one plan per block product, one ContractGroup per wave."""

    def __init__(self, C: BlockSparseTensor, A: BlockSparseTensor, indA, B: BlockSparseTensor, indB, indC, *,
                 conjA=False, conjB=False, method="auto", mode="persistent", graph=False):
        from . import ContractGroup, plan_contract
        prods, c_spaces = pair_blocks(A.spaces, A.keys, indA, B.spaces, B.keys, indB, indC)
        if tuple(c_spaces) != C.spaces:
            raise _abi.DimensionMismatch("C's legs differ from the free legs of A and B")
        keys_c = set(C.keys)
        prods = [p for p in prods if p.kc in keys_c]   # others have no C block (flux mismatch)
        self.C, self.A, self.B = C, A, B
        self.waves = waves_of(prods)
        self.plans = [[plan_contract(C.block(p.kc), A.block(p.ka), tuple(indA), B.block(p.kb), tuple(indB),
                                     tuple(indC), conjA=conjA, conjB=conjB, method=method) for p in wave]
                      for wave in self.waves]
        self.groups = [ContractGroup(ps, mode=mode, graph=graph) for ps in self.plans]
        touched = {p.kc for p in prods}
        self.untouched = [k for k in C.keys if k not in touched]
        self.flops = sum((8.0 if C.dtype.is_complex else 2.0) * float(np.prod(A.block_shape(p.ka))) *
                         float(np.prod(B.block_shape(p.kb))) /
                         float(np.prod([A.block_shape(p.ka)[i] for i, l in enumerate(indA) if l in indB]) or 1)
                         for p in prods)
        self.products = len(prods)

    def execute(self, alpha=1.0, beta=0.0, stream=None) -> BlockSparseTensor:
        from . import add_trace
        for w, g in enumerate(self.groups):
            n = len(self.plans[w])
            g.execute([alpha] * n, [beta if w == 0 else 1.0] * n, stream=stream)
        if complex(beta) != 1.0:
            for k in self.untouched:
                v = self.C.block(k)
                lab = tuple(range(1, v.ndim + 1))
                add_trace(v, 0.0, v, lab, beta, lab, stream=stream)   # C = beta * C, A not read
        return self.C

    def release(self) -> None:
        for g in self.groups:
            g.release()
        for ps in self.plans:
            for p in ps:
                p.release()


def contract(A: BlockSparseTensor, indA, B: BlockSparseTensor, indB, indC, *, alpha=1.0, beta=0.0,
             C: Optional[BlockSparseTensor] = None, conjA=False, conjB=False, method="auto",
             mode="persistent") -> BlockSparseTensor:
    """One-shot block-sparse contraction; C is created (flux = A.flux + B.flux)
    when not given.  Waits for the work."""
    if C is None:
        _, c_spaces = pair_blocks(A.spaces, A.keys, indA, B.spaces, B.keys, indB, indC)
        C = BlockSparseTensor(c_spaces, A.flux + B.flux, A.dtype, A.buffer.device)
    bc = BlockContraction(C, A, indA, B, indB, indC, conjA=conjA, conjB=conjB, method=method, mode=mode)
    bc.execute(alpha, beta)
    torch.cuda.synchronize()
    bc.release()
    return C
