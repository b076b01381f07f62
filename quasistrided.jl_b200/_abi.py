"""ctypes binding of include/qsgpu.h (libqsgpu.so) and status -> exception mapping."""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libqsgpu.so")

QS_OK, QS_EINVAL, QS_EDIM, QS_EBOUNDS, QS_ENOMEM, QS_ETIMEOUT, QS_ECUDA, QS_ENOTSUP = range(8)
QS_F32, QS_F64, QS_C32, QS_C64 = range(4)
QS_OP = {"identity": 0, "conj": 1, "transpose": 2, "adjoint": 3}
QS_ACC = {None: 0, "Float32": 1, "Float64": 2}
QS_METHOD = {"auto": 0, "native": 1, "ozaki": 2, "bf16x3": 3}
QS_METHOD_NAME = {v: k for k, v in QS_METHOD.items()}
QS_MODE = {"auto": 0, "never": 1, "always": 2}
QS_PATH_NAME = {0: "EmptyPath", 1: "ScalePath", 2: "DotPath", 3: "OuterPath", 4: "NestPath"}
QS_CPLX = {None: 0, "planar": 1, "1m": 2}
QS_PLAN_HOST_ONLY = 1
QS_PLAN_BATCH_LABELS = 8
QS_PLAN_OZ_SINGLE_SM = 16

ELTYPE_NAME = {QS_F32: "Float32", QS_F64: "Float64", QS_C32: "ComplexF32", QS_C64: "ComplexF64"}


class ArgumentError(ValueError):
    """Julia's ArgumentError: invalid labels, eltypes, conjugated C, aliasing."""


class DimensionMismatch(ValueError):
    """Julia's DimensionMismatch: a label's axis lengths differ."""


class BoundsError(IndexError):
    """Julia's BoundsError: a view reaches outside its parent storage."""


class EngineError(RuntimeError):
    """A device-side failure (CUDA error, allocation failure, timeout)."""


class DeviceTimeout(EngineError):
    """A bounded device wait of a tensor-core kernel gave up (QS_ETIMEOUT):
    the kernel stopped without writing C; the GPU and the plan stay usable."""


class qs_view(ctypes.Structure):
    _fields_ = [
        ("data", ctypes.c_void_p),
        ("length", ctypes.c_int64),
        ("offset", ctypes.c_int64),
        ("size", ctypes.POINTER(ctypes.c_int64)),
        ("strides", ctypes.POINTER(ctypes.c_int64)),
        ("ndim", ctypes.c_int32),
        ("eltype", ctypes.c_int32),
        ("op", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class qs_plan_options(ctypes.Structure):
    _fields_ = [
        ("conjA", ctypes.c_int32),
        ("conjB", ctypes.c_int32),
        ("accumulator", ctypes.c_int32),
        ("method", ctypes.c_int32),
        ("m_block", ctypes.c_int64),
        ("k_block", ctypes.c_int64),
        ("n_block", ctypes.c_int64),
        ("dot_mode", ctypes.c_int32),
        ("outer_mode", ctypes.c_int32),
        ("unpacked_b_mode", ctypes.c_int32),
        ("ozaki_slices", ctypes.c_int32),
        ("complex_mode", ctypes.c_int32),
        ("flags", ctypes.c_int32),
        ("native_tile", ctypes.c_int32),
        ("allocator", ctypes.c_void_p),
    ]


ALLOC_FN = ctypes.CFUNCTYPE(ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t)
FREE_FN = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p)


class qs_allocator(ctypes.Structure):
    _fields_ = [
        ("ctx", ctypes.c_void_p),
        ("alloc", ALLOC_FN),
        ("free", FREE_FN),
    ]


class qs_plan_info(ctypes.Structure):
    _fields_ = [
        ("path", ctypes.c_int32),
        ("method", ctypes.c_int32),
        ("compute_type", ctypes.c_int32),
        ("swapped", ctypes.c_int32),
        ("conjA", ctypes.c_int32),
        ("conjB", ctypes.c_int32),
        ("ozaki_slices", ctypes.c_int32),
        ("complex_mode", ctypes.c_int32),
        ("m_length", ctypes.c_int64),
        ("n_length", ctypes.c_int64),
        ("k_length", ctypes.c_int64),
        ("m_rank", ctypes.c_int32),
        ("n_rank", ctypes.c_int32),
        ("k_rank", ctypes.c_int32),
        ("bounds_ok", ctypes.c_int32),
        ("m_labels", ctypes.c_int64 * 16),
        ("n_labels", ctypes.c_int64 * 16),
        ("k_labels", ctypes.c_int64 * 16),
        ("workspace_bytes", ctypes.c_int64),
        ("stride_class", ctypes.c_int32),
        ("native_tile", ctypes.c_int32),
        ("batch_rank", ctypes.c_int32),
        ("batch_length", ctypes.c_int64),
        ("batch_labels", ctypes.c_int64 * 16),
    ]


class qs_group_info(ctypes.Structure):
    _fields_ = [
        ("nplans", ctypes.c_int32),
        ("launches", ctypes.c_int32),
        ("native_plans", ctypes.c_int32),
        ("tc_plans", ctypes.c_int32),
        ("single_plans", ctypes.c_int32),
        ("classes", ctypes.c_int32),
        ("tiles", ctypes.c_int64),
        ("table_bytes", ctypes.c_int64),
    ]


QS_GROUP_PERSISTENT = 0
QS_GROUP_SEQUENTIAL = 1
QS_GROUP_GRAPH = 2

# Every symbol the header declares, with its ctypes signature.
_P = ctypes.c_void_p
_I64P = ctypes.POINTER(ctypes.c_int64)
_DP = ctypes.POINTER(ctypes.c_double)
SIGNATURES = {
    "qs_plan_contract": (ctypes.c_int, [ctypes.POINTER(_P), ctypes.POINTER(qs_view), ctypes.POINTER(qs_view), _I64P,
                                        ctypes.POINTER(qs_view), _I64P, _I64P, ctypes.POINTER(qs_plan_options)]),
    "qs_execute": (ctypes.c_int, [_P, _DP, _DP, _P]),
    "qs_contract": (ctypes.c_int, [ctypes.POINTER(qs_view), _DP, ctypes.POINTER(qs_view), _I64P,
                                   ctypes.POINTER(qs_view), _I64P, _DP, _I64P, ctypes.POINTER(qs_plan_options), _P]),
    "qs_plan_destroy": (ctypes.c_int, [_P]),
    "qs_plan_get_info": (ctypes.c_int, [_P, ctypes.POINTER(qs_plan_info)]),
    "qs_plan_rebind": (ctypes.c_int, [_P, _P, _P, _P]),
    "qs_contraction_labels": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _I64P, _I64P, _I64P,
                                             _I64P, _I64P, _I64P]),
    "qs_execute_grouped": (ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(_P), _DP, _DP, _P]),
    "qs_group_create": (ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(_P), ctypes.c_int32, ctypes.POINTER(_P)]),
    "qs_group_execute": (ctypes.c_int, [_P, _DP, _DP, _P]),
    "qs_group_get_info": (ctypes.c_int, [_P, ctypes.POINTER(qs_group_info)]),
    "qs_group_destroy": (ctypes.c_int, [_P]),
    "qs_last_error": (ctypes.c_size_t, [ctypes.c_char_p, ctypes.c_size_t]),
    "qs_launch_count": (ctypes.c_int64, []),
    "qs_plan_profile": (ctypes.c_int, [_P, ctypes.c_int32]),
    "qs_plan_stage_times": (ctypes.c_int, [_P, _DP, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                           ctypes.POINTER(ctypes.c_int32)]),
    "qs_plan_check_status": (ctypes.c_int, [_P, _P]),
    "qs_plan_set_wait_limit": (ctypes.c_int, [_P, ctypes.c_uint64, ctypes.c_int32]),
    "qs_contract_noalloc": (ctypes.c_int, [ctypes.POINTER(qs_view), _DP, ctypes.POINTER(qs_view), _I64P,
                                           ctypes.POINTER(qs_view), _I64P, _DP, _I64P,
                                           ctypes.POINTER(qs_plan_options), _P]),
    "qs_tensoradd_trace": (ctypes.c_int, [ctypes.POINTER(qs_view), _DP, ctypes.POINTER(qs_view), _I64P,
                                          ctypes.c_int32, _DP, _I64P, _P]),
    "qs_version": (ctypes.c_char_p, []),
    "qs_arena_create": (ctypes.c_int, [ctypes.POINTER(_P), _P, ctypes.c_size_t]),
    "qs_arena_destroy": (ctypes.c_int, [_P]),
    "qs_arena_allocator": (_P, [_P]),
    "qs_arena_alloc": (ctypes.c_int, [_P, ctypes.c_size_t, ctypes.POINTER(_P)]),
    "qs_arena_free": (ctypes.c_int, [_P, _P, ctypes.c_size_t, _P]),
    "qs_arena_checkpoint": (ctypes.c_size_t, [_P]),
    "qs_arena_reset": (ctypes.c_int, [_P, ctypes.c_size_t, _P]),
    "qs_arena_get_info": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t),
                                         ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_int64)]),
}

_lib = None


def lib():
    """Load libqsgpu.so (built in-tree); fails loudly when it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise EngineError(
                f"libqsgpu.so is not built ({LIB_PATH}); run quasistrided.jl_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    buf = ctypes.create_string_buffer(4096)
    lib().qs_last_error(buf, 4096)
    return buf.value.decode(errors="replace")


def check(rc: int) -> None:
    if rc == QS_OK:
        return
    msg = last_error()
    if rc == QS_EINVAL or rc == QS_ENOTSUP:
        raise ArgumentError(msg)
    if rc == QS_EDIM:
        raise DimensionMismatch(msg)
    if rc == QS_EBOUNDS:
        raise BoundsError(msg)
    if rc == QS_ETIMEOUT:
        raise DeviceTimeout(f"status {rc}: {msg}")
    raise EngineError(f"status {rc}: {msg}")
