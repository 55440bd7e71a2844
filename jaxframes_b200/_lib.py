"""ctypes binding of ``libjfx.so`` (declarations: ``include/jfx.h``).

The library is the only compute path: if it is missing, or no CUDA device is
present, every call raises ``JfxUnavailable``.  There is no CPU fallback.
"""

from __future__ import annotations

import ctypes
import os
import threading

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libjfx.so")

JFX_OK = 0
STATUS_NAMES = {
    -1: "JFX_ERR_ARG", -2: "JFX_ERR_DTYPE", -3: "JFX_ERR_ALLOC",
    -4: "JFX_ERR_TIMEOUT", -5: "JFX_ERR_CAPACITY", -6: "JFX_ERR_CUDA",
}

I8, I16, I32, I64, U8, U16, U32, U64, F32, F64, BOOL = range(1, 12)
TORCH_TO_JFX = {
    torch.int8: I8, torch.int16: I16, torch.int32: I32, torch.int64: I64,
    torch.uint8: U8, torch.uint16: U16, torch.uint32: U32, torch.uint64: U64,
    torch.float32: F32, torch.float64: F64, torch.bool: BOOL,
}
JFX_TO_TORCH = {v: k for k, v in TORCH_TO_JFX.items()}

COL_DESC = 1
AGG_SUM, AGG_MEAN, AGG_COUNT, AGG_MIN, AGG_MAX = 1, 2, 4, 8, 16
AGG_BITS = {"sum": AGG_SUM, "mean": AGG_MEAN, "count": AGG_COUNT, "min": AGG_MIN, "max": AGG_MAX}
JOIN_KINDS = {"inner": 0, "left": 1, "right": 2, "outer": 3}
WS_SORT, WS_GROUPBY, WS_JOIN, WS_PARTITION, WS_LEARNED, WS_BATCH = 1, 2, 3, 4, 5, 6
SORT_STATIC_MAX_ROWS = 524288  # JFX_SORT_STATIC_MAX_ROWS


class JfxUnavailable(RuntimeError):
    """The CUDA extension cannot run here (library missing or no GPU)."""


class JfxError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class Column(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("dtype", ctypes.c_int32), ("flags", ctypes.c_uint32)]


class AggColumn(ctypes.Structure):
    _fields_ = [
        ("data", ctypes.c_void_p), ("dtype", ctypes.c_int32), ("aggs", ctypes.c_uint32),
        ("out_sum", ctypes.c_void_p), ("out_mean", ctypes.c_void_p), ("out_count", ctypes.c_void_p),
        ("out_min", ctypes.c_void_p), ("out_max", ctypes.c_void_p),
        ("mean_dtype", ctypes.c_int32), ("count_dtype", ctypes.c_int32),
    ]


class Tuning(ctypes.Structure):
    _fields_ = [("max_digit_bits", ctypes.c_int32), ("two_phase", ctypes.c_int32),
                ("spin_limit_us", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class Fault(ctypes.Structure):
    _fields_ = [("withhold_tile", ctypes.c_int32), ("learned_fallback", ctypes.c_int32),
                ("fail_workspace", ctypes.c_int32), ("withhold_order", ctypes.c_int32)]


class JoinPayload(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("n", ctypes.c_int64), ("dtype", ctypes.c_int32),
                ("side", ctypes.c_int32), ("out", ctypes.c_void_p), ("out_dtype", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class JoinPlan(ctypes.Structure):
    _fields_ = [("opaque", ctypes.c_uint64 * 160)]


_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_INT = ctypes.c_int
_SIZE = ctypes.c_size_t

# exported symbol -> (restype, argtypes); must match include/jfx.h
SIGNATURES = {
    "jfx_last_error": (ctypes.c_char_p, []),
    "jfx_version": (_INT, []),
    "jfx_max_rows": (_INT, []),
    "jfx_workspace_size": (_SIZE, [_INT, _I64, _I64]),
    "jfx_sort": (_INT, [ctypes.POINTER(Column), _I64, _INT, _P, _P, _P, _SIZE, _P]),
    "jfx_sort_static": (_INT, [ctypes.POINTER(Column), _I64, _INT, _P, _P, _P]),
    "jfx_lexsort": (_INT, [ctypes.POINTER(Column), _INT, _I64, _P, _P, _SIZE, _P]),
    "jfx_groupby": (_INT, [ctypes.POINTER(Column), _INT, _I64, _INT, ctypes.POINTER(AggColumn), _INT,
                           ctypes.POINTER(_P), ctypes.POINTER(_I64), _P, _SIZE, _P]),
    "jfx_join_prepare": (_INT, [ctypes.POINTER(Column), _I64, ctypes.POINTER(Column), _I64, _INT, _INT,
                                ctypes.POINTER(JoinPlan), ctypes.POINTER(_I64), _P, _SIZE, _P]),
    "jfx_join_expand": (_INT, [ctypes.POINTER(JoinPlan), _P, _P, ctypes.POINTER(_P), _P]),
    "jfx_join_prepare_payloads": (_INT, [ctypes.POINTER(Column), _I64, ctypes.POINTER(Column), _I64, _INT, _INT,
                                         ctypes.POINTER(JoinPayload), _INT, ctypes.POINTER(JoinPlan),
                                         ctypes.POINTER(_I64), _P, _SIZE, _P]),
    "jfx_join_expand_gather": (_INT, [ctypes.POINTER(JoinPlan), _P, _P, ctypes.POINTER(_P),
                                      ctypes.POINTER(JoinPayload), _INT, _P]),
    "jfx_join_unmatched": (_INT, [ctypes.POINTER(JoinPlan), _INT, _P, _I64, ctypes.POINTER(_I64), _P]),
    "jfx_coalesce": (_INT, [_P, _P, _I64, _P, _P, _I64, _I64, ctypes.c_int32, _P, _P]),
    "jfx_gather": (_INT, [_P, ctypes.c_int32, _I64, _P, _I64, _P, ctypes.c_int32, _P]),
    "jfx_hash_columns": (_INT, [ctypes.POINTER(Column), _INT, _I64, _P, _P]),
    "jfx_hash_partition": (_INT, [ctypes.POINTER(Column), _INT, _I64, _INT, _P, _P, _P, _P, _SIZE, _P]),
    "jfx_learned_sort": (_INT, [_P, _I64, _P, _P, _INT, ctypes.POINTER(ctypes.c_int32), _P, _SIZE, _P]),
    "jfx_batch_partition_groupby": (_INT, [_P, _P, _P, _INT, _I64, _INT, _INT, _P, _P, _P, _P, _P, _P, _P, _P,
                                           _SIZE, _P]),
    "jfx_batch_status": (_INT, [_P, _SIZE, _P]),
    "jfx_set_tuning": (_INT, [ctypes.POINTER(Tuning)]),
    "jfx_get_tuning": (_INT, [ctypes.POINTER(Tuning)]),
    "jfx_set_fault": (_INT, [ctypes.POINTER(Fault)]),
    "jfx_launch_count": (ctypes.c_uint64, []),
    "jfx_timing_enable": (_INT, [_INT]),
    "jfx_timing_read": (_INT, [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_I64),
                               ctypes.POINTER(ctypes.c_double)]),
}

_lock = threading.Lock()
_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads libjfx.so and declares every exported signature (no GPU needed)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise JfxUnavailable(f"{path} is missing; build it with `python -m jaxframes_b200.build`")
        lib = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def lib() -> ctypes.CDLL:
    """The library, for a compute call: requires a CUDA device."""
    if not torch.cuda.is_available():
        raise JfxUnavailable("no CUDA device: the jfx kernels need a B200 (sm_100a); there is no CPU fallback")
    return load_library()


def check(status: int) -> None:
    if status != JFX_OK:
        msg = _lib.jfx_last_error().decode(errors="replace") if _lib else ""
        raise JfxError(status, msg)


def stream_handle(device=None) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def jfx_dtype(t: torch.Tensor) -> int:
    try:
        return TORCH_TO_JFX[t.dtype]
    except KeyError:
        raise TypeError(f"unsupported dtype {t.dtype}") from None


def column(t: torch.Tensor, flags: int = 0) -> Column:
    return Column(t.data_ptr(), jfx_dtype(t), flags)


def workspace(kind: int, n1: int, n2: int = 0, device=None) -> torch.Tensor:
    size = load_library().jfx_workspace_size(kind, n1, n2)
    return torch.empty(max(size, 256), dtype=torch.uint8, device=device or "cuda")
