"""ctypes wrapper of the oracle (oracle/oracle.c) — test infrastructure only.

Used by tests/, __graft_entry__.smoke() and bench.py's CPU arm as the
checker/baseline; the engine never calls it.  Operands are host numpy
arrays wrapped as ``HostView`` (parent, size, strides, offset, op), the same
fields as the engine's StridedView.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_ET = {np.dtype(np.float32): 0, np.dtype(np.float64): 1, np.dtype(np.complex64): 2,
       np.dtype(np.complex128): 3}
_OP = {"identity": 0, "conj": 1, "transpose": 2, "adjoint": 3}


class or_view(ctypes.Structure):
    _fields_ = [
        ("data", ctypes.c_void_p), ("length", ctypes.c_int64), ("offset", ctypes.c_int64),
        ("size", ctypes.POINTER(ctypes.c_int64)), ("strides", ctypes.POINTER(ctypes.c_int64)),
        ("ndim", ctypes.c_int32), ("eltype", ctypes.c_int32), ("op", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


def lib():
    global _LIB
    if _LIB is None:
        from . import build as _b  # type: ignore
        path = _b.build()
        L = ctypes.CDLL(path)
        P = ctypes.POINTER
        L.oracle_brute.restype = ctypes.c_int
        L.oracle_brute.argtypes = [P(or_view), P(ctypes.c_double), P(or_view), P(ctypes.c_int64),
                                   P(or_view), P(ctypes.c_int64), P(ctypes.c_double), P(ctypes.c_int64),
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, P(ctypes.c_int64), ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int64, ctypes.c_int64, ctypes.c_int]
        L.oracle_nest_f64.restype = ctypes.c_int
        L.oracle_nest_f64.argtypes = [P(or_view), ctypes.c_double, P(or_view), P(ctypes.c_int64),
                                      P(or_view), P(ctypes.c_int64), ctypes.c_double, P(ctypes.c_int64),
                                      ctypes.c_int64, ctypes.c_int64, ctypes.c_int]
        L.oracle_max_threads.restype = ctypes.c_int
        _LIB = L
    return _LIB


class HostView:
    """A strided window into a flat host numpy array."""

    def __init__(self, parent: np.ndarray, size: Sequence[int], strides: Sequence[int],
                 offset: int = 0, op: str = "identity"):
        assert parent.ndim == 1 and parent.flags.c_contiguous
        self.parent = parent
        self.size = tuple(int(s) for s in size)
        self.strides = tuple(int(s) for s in strides)
        self.offset = int(offset)
        self.op = op

    @property
    def ndim(self):
        return len(self.size)

    def _c(self, keep):
        sz = (ctypes.c_int64 * max(1, self.ndim))(*self.size)
        st = (ctypes.c_int64 * max(1, self.ndim))(*self.strides)
        keep += [sz, st]
        v = or_view()
        v.data = self.parent.ctypes.data
        v.length = self.parent.size
        v.offset = self.offset
        v.size, v.strides = sz, st
        v.ndim = self.ndim
        v.eltype = _ET[self.parent.dtype]
        v.op = _OP[self.op]
        return v

    def to_array(self) -> np.ndarray:
        """The window as a dense numpy array (op applied)."""
        itm = self.parent.itemsize
        a = np.lib.stride_tricks.as_strided(self.parent[self.offset:] if all(s >= 0 for s in self.strides)
                                            else self.parent, shape=self.size,
                                            strides=[s * itm for s in self.strides])
        if not all(s >= 0 for s in self.strides):
            idx = np.zeros(self.size, dtype=np.int64) + self.offset
            for d, (n, s) in enumerate(zip(self.size, self.strides)):
                shp = [1] * self.ndim
                shp[d] = n
                idx = idx + (np.arange(n) * s).reshape(shp)
            a = self.parent[idx]
        a = np.array(a)
        if self.op in ("conj", "adjoint") and np.iscomplexobj(a):
            a = a.conj()
        return a


def colmajor(shape, dtype=np.float64, data: Optional[np.ndarray] = None) -> HostView:
    n = int(np.prod(shape)) if len(shape) else 1
    parent = np.zeros(max(n, 1), dtype=dtype) if data is None else np.ascontiguousarray(data, dtype=dtype).reshape(-1)
    st, acc = [], 1
    for s in shape:
        st.append(acc)
        acc *= int(s)
    return HostView(parent, shape, st, 0)


def _labels(ind, keep):
    arr = (ctypes.c_int64 * max(1, len(ind)))(*[int(x) for x in ind])
    keep.append(arr)
    return arr


def brute(C: HostView, alpha, A: HostView, indA, B: HostView, indB, beta, indC, *,
          conjA=False, conjB=False, accumulator=None, korder=None, precision=0,
          c_range=(0, -1), threads=None) -> HostView:
    """C = alpha*sum A*B + beta*C by brute force over label assignments, in place."""
    keep: list = []
    za, zb = complex(alpha), complex(beta)
    al = (ctypes.c_double * 2)(za.real, za.imag)
    be = (ctypes.c_double * 2)(zb.real, zb.imag)
    acc = {None: 0, "Float32": 1, "Float64": 2}[accumulator]
    ko = _labels(korder, keep) if korder else None
    nthreads = threads or min(8, lib().oracle_max_threads())
    rc = lib().oracle_brute(ctypes.byref(C._c(keep)), al, ctypes.byref(A._c(keep)), _labels(indA, keep),
                            ctypes.byref(B._c(keep)), _labels(indB, keep), be, _labels(indC, keep),
                            int(conjA), int(conjB), acc, ko, len(korder) if korder else 0, precision,
                            c_range[0], c_range[1], nthreads)
    if rc != 0:
        raise ValueError(f"oracle_brute: malformed input ({rc})")
    return C


def nest_f64(C: HostView, alpha, A: HostView, indA, B: HostView, indB, beta, indC, *,
             m_range=(0, -1), threads=None) -> HostView:
    """The five-loop nest restatement (real Float64), in place."""
    keep: list = []
    nthreads = threads or lib().oracle_max_threads()
    rc = lib().oracle_nest_f64(ctypes.byref(C._c(keep)), float(alpha), ctypes.byref(A._c(keep)),
                               _labels(indA, keep), ctypes.byref(B._c(keep)), _labels(indB, keep),
                               float(beta), _labels(indC, keep), m_range[0], m_range[1], nthreads)
    if rc != 0:
        raise ValueError(f"oracle_nest_f64: malformed input ({rc})")
    return C


def max_threads() -> int:
    return lib().oracle_max_threads()


def label_subview(v: HostView, labels, picks: dict) -> HostView:
    """The sub-view of `v` (axes labelled `labels`) that keeps, for every
    label in `picks` (label -> (start, step, count)), the indices start,
    start + step, ..., start + (count - 1) * step of that label's axis.  A
    contraction over such sub-views of A, B and C computes exactly the picked
    elements of C: a sample spread over every index of C for the checker."""
    size, strides, offset = list(v.size), list(v.strides), v.offset
    for d, lab in enumerate(labels):
        if lab in picks:
            start, step, count = picks[lab]
            assert 0 <= start and start + (count - 1) * step < size[d]
            offset += start * strides[d]
            strides[d] *= step
            size[d] = count
    return HostView(v.parent, size, strides, offset, v.op)


def rel_fro(got: np.ndarray, ref: np.ndarray) -> float:
    """Relative Frobenius error ||got - ref|| / ||ref||, accumulated in
    extended precision."""
    ref = np.asarray(ref, dtype=np.complex256 if np.iscomplexobj(ref) else np.longdouble)
    d = np.linalg.norm((np.asarray(got, dtype=ref.dtype) - ref).ravel())
    n = np.linalg.norm(ref.ravel())
    return float(d / n) if n > 0 else float(d)
