"""Helpers for the GPU parity tests: paired host (oracle) / device (engine)
operands with identical layout and values, and the error measures."""
from __future__ import annotations

import numpy as np
import torch

from oracle.oracle import HostView

NP = {"Float32": np.float32, "Float64": np.float64, "ComplexF32": np.complex64,
      "ComplexF64": np.complex128}
TORCH = {"Float32": torch.float32, "Float64": torch.float64, "ComplexF32": torch.complex64,
         "ComplexF64": torch.complex128}


def randn(rng, n, et):
    if et.startswith("Complex"):
        v = (rng.standard_normal(n) + 1j * rng.standard_normal(n)) / np.sqrt(2)
    else:
        v = rng.standard_normal(n)
    return v.astype(NP[et])


class Pair:
    """The same strided view on the host (HostView) and on the device (StridedView)."""

    def __init__(self, qs, parent: np.ndarray, size, strides, offset=0, op="identity"):
        self.host = HostView(np.ascontiguousarray(parent).copy(), size, strides, offset, op)
        self.dev = qs.StridedView(torch.from_numpy(parent.copy()).cuda(), size, strides, offset, op)

    def device_parent(self) -> np.ndarray:
        return self.dev.parent.cpu().numpy()


def colmajor_pair(qs, rng, shape, et, fill=None, op="identity"):
    n = int(np.prod(shape)) if len(shape) else 1
    parent = randn(rng, max(n, 1), et) if fill is None else np.full(max(n, 1), fill, dtype=NP[et])
    st, acc = [], 1
    for s in shape:
        st.append(acc)
        acc *= s
    return Pair(qs, parent, shape, st, 0, op)


def rel_fro(got: np.ndarray, ref: np.ndarray) -> float:
    ref = np.asarray(ref, dtype=np.complex256 if np.iscomplexobj(ref) else np.float64)
    d = np.linalg.norm((np.asarray(got, dtype=ref.dtype) - ref).ravel())
    n = np.linalg.norm(ref.ravel())
    return float(d / n) if n > 0 else float(d)


def run_pair(qs, orc, C: Pair, alpha, A: Pair, indA, B: Pair, indB, beta, indC, *,
             precision=0, **plankw):
    """Execute the engine on the device and the oracle on the host (in the
    plan's K order); returns (device C parent, oracle C parent, plan)."""
    plan = qs.plan_contract(C.dev, A.dev, indA, B.dev, indB, indC, **plankw)
    qs.execute(plan, alpha, beta)
    torch.cuda.synchronize()
    orc.brute(C.host, alpha, A.host, indA, B.host, indB, beta, indC,
              conjA=plankw.get("conjA", False), conjB=plankw.get("conjB", False),
              accumulator=plankw.get("accumulator"), korder=list(plan.k_labels) or None,
              precision=precision)
    return C.device_parent(), C.host.parent, plan
