"""Loads the in-tree CUDA library and declares its C ABI (include/spk_b200.h).

The product path has no CPU fallback: if libspk_b200.so is missing or cannot
be loaded, every call fails loudly with SpkUnavailable.
"""

from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("SPK_LIBRARY") or os.path.join(HERE, "libspk_b200.so")


class SpkUnavailable(RuntimeError):
    """The CUDA extension is missing or no usable GPU is present."""


class SpkError(RuntimeError):
    def __init__(self, status: int, code: str, where: str = ""):
        super().__init__(f"{where}: {code} ({status})" if where else f"{code} ({status})")
        self.status = status
        self.code = code


class CorrelationSpec(ctypes.Structure):
    _fields_ = [("environment_shape", ctypes.c_uint32 * 3), ("kernel_shape", ctypes.c_uint32 * 3),
                ("environment_first", ctypes.c_int64 * 3), ("kernel_first", ctypes.c_int64 * 3)]


class CorrelationLimits(ctypes.Structure):
    _fields_ = [("max_working_bytes", ctypes.c_uint64), ("reserved_bytes", ctypes.c_uint64),
                ("max_padded_cells", ctypes.c_uint64), ("max_direct_terms", ctypes.c_uint64)]


class CorrelationResultC(ctypes.Structure):
    _fields_ = [("translation_first", ctypes.c_int64 * 3), ("shape", ctypes.c_uint32 * 3),
                ("max_integer_residual", ctypes.c_double), ("mass_residual", ctypes.c_double),
                ("max_probe_error", ctypes.c_double), ("padded_cells", ctypes.c_uint64),
                ("working_bytes_peak", ctypes.c_uint64), ("direct_terms", ctypes.c_uint64),
                ("padded_shape", ctypes.c_uint32 * 3)]


class CorrelationEstimateC(ctypes.Structure):
    _fields_ = [("padded_shape", ctypes.c_uint32 * 3), ("padded_cells", ctypes.c_uint64),
                ("working_bytes", ctypes.c_uint64)]


class Control(ctypes.Structure):
    _fields_ = [("stop_word", ctypes.POINTER(ctypes.c_uint32)), ("deadline_ns", ctypes.c_int64)]


_lib = None


def lib():
    """The loaded library; raises SpkUnavailable when it cannot be loaded."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise SpkUnavailable(f"{LIB_PATH} is missing: run python cpp-max-packer_b200/build.py")
    try:
        handle = ctypes.CDLL(LIB_PATH)
    except OSError as exc:  # pragma: no cover - environment specific
        raise SpkUnavailable(str(exc)) from exc
    _declare(handle)
    _lib = handle
    return handle


def _declare(h):
    P = ctypes.c_void_p
    h.spk_status_code.restype = ctypes.c_char_p
    h.spk_status_code.argtypes = [ctypes.c_int]
    h.spk_context_create.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(P)]
    h.spk_context_destroy.argtypes = [P]
    h.spk_context_destroy.restype = None
    h.spk_context_launches.argtypes = [P]
    h.spk_context_launches.restype = ctypes.c_uint64
    h.spk_context_stream.argtypes = [P]
    h.spk_context_stream.restype = ctypes.c_void_p
    h.spk_context_set_profiling.argtypes = [P, ctypes.c_int]
    h.spk_context_pass_times.argtypes = [P, P, P, ctypes.c_uint32]
    h.spk_context_pass_bytes.argtypes = [P, P, ctypes.c_uint32]
    h.spk_estimate_correlation.argtypes = [ctypes.POINTER(CorrelationSpec), ctypes.c_uint32,
                                           ctypes.POINTER(CorrelationEstimateC)]
    for name in ("spk_correlate_binary", "spk_correlate_proximity"):
        getattr(h, name).argtypes = [P, ctypes.POINTER(CorrelationSpec), P, P, ctypes.POINTER(CorrelationLimits),
                                     ctypes.POINTER(Control), ctypes.c_uint32, P, ctypes.c_uint64,
                                     ctypes.POINTER(CorrelationResultC)]
    h.spk_correlate_binary_mask.argtypes = [P, ctypes.POINTER(CorrelationSpec), P, P,
                                            ctypes.POINTER(CorrelationLimits), ctypes.POINTER(Control),
                                            ctypes.c_uint32, ctypes.POINTER(ctypes.c_int64),
                                            ctypes.POINTER(ctypes.c_uint32), ctypes.c_uint32, P, ctypes.c_uint64,
                                            ctypes.POINTER(CorrelationResultC)]
    h.spk_build_proximity.argtypes = [P, P, P, P]
    h.spk_build_proximity_static.argtypes = [P, P, P, P]
    h.spk_check_bounded_wait.argtypes = [P, ctypes.c_uint32]


def status_code(status: int) -> str:
    return lib().spk_status_code(status).decode()


def check(status: int, where: str = ""):
    if status:
        raise SpkError(status, status_code(status), where)
