"""Host mirror of the reference's compute::correlate_* API on the B200 path.

Reference interface (engine/pack_compute/include/spectrapack/compute/
correlation.hpp:22-117): ``correlate_binary_cpu(spec, environment, kernel,
limits, control)`` and ``correlate_proximity_cpu(...)`` return either a
CorrelationResult (translation_first, shape, values, numeric report, stats)
or a CorrelationFailure (static code, message, stats); they never throw.
``correlate_binary`` / ``correlate_proximity`` here keep those names'
meaning, argument order and error behaviour, and run on the GPU through the
C ABI; ``precision`` selects FP64 (the reference's tolerances hold) or FP32.
"""

from __future__ import annotations

import ctypes
import dataclasses
import time
from typing import Optional, Sequence, Union

import numpy as np

from . import _lib
from ._lib import SpkError, check, lib

FP32 = 0
FP64 = 1
FP16 = 2  # FP32 transforms, joint spectrum stored in FP16 before the product
MASK_ZERO = 0  # spk_correlate_binary_mask: mark translations with a zero overlap count
MASK_NONZERO = 1  # ... or with a non-zero one

_MESSAGES = {
    "CORRELATION_SHAPE_OVERFLOW": "Correlation extents must be positive and representable.",
    "CORRELATION_INDEX_OVERFLOW": "The first output translation is not representable.",
    "CORRELATION_INVALID_FIELD": "Shape does not match supplied cells.",
    "CORRELATION_INVALID_ENVIRONMENT": "Environment cells must be finite values in [0,1].",
    "CORRELATION_INVALID_KERNEL": "Kernel cells must be binary.",
    "CORRELATION_NUMERIC_RANGE": "Correlation mass is not exactly representable.",
    "CORRELATION_PADDED_CELL_LIMIT": "Padded field exceeds its cell limit.",
    "CORRELATION_MEMORY_LIMIT": "Correlation buffers exceed their memory limit.",
    "CORRELATION_NUMERIC": "FFT output failed a numeric check.",
    "CORRELATION_DIRECT_TERM_LIMIT": "Deterministic direct checks exhausted their work limit.",
    "CORRELATION_ALLOCATION": "Correlation allocation failed.",
    "OPERATION_CANCELLED": "Correlation interrupted.",
    "DEADLINE_EXCEEDED": "Correlation interrupted.",
}


@dataclasses.dataclass
class CorrelationSpec:
    """X-fastest fields; kernel cell i sits at translation + kernel_first + i."""

    environment_shape: Sequence[int]
    kernel_shape: Sequence[int]
    environment_first: Sequence[int] = (0, 0, 0)
    kernel_first: Sequence[int] = (0, 0, 0)


@dataclasses.dataclass
class CorrelationLimits:
    max_working_bytes: int = 512 << 20
    reserved_bytes: int = 0
    max_padded_cells: int = 16_777_216
    max_direct_terms: int = 200_000_000


@dataclasses.dataclass
class NumericReport:
    max_integer_residual: float = 0.0
    mass_residual: float = 0.0
    max_probe_error: float = 0.0


@dataclasses.dataclass
class CorrelationStats:
    padded_cells: int = 0
    working_bytes_peak: int = 0
    direct_terms: int = 0


@dataclasses.dataclass
class CorrelationResult:
    translation_first: tuple
    shape: tuple
    values: np.ndarray
    numeric: NumericReport
    stats: CorrelationStats
    padded_shape: tuple = (0, 0, 0)


@dataclasses.dataclass
class MaskResult:
    """spk_correlate_binary_mask's outcome: the correlation range and checks as
    in CorrelationResult, and the u8 mask over the requested box (X fastest)."""
    translation_first: tuple
    shape: tuple
    box_first: tuple
    box_shape: tuple
    mask: np.ndarray
    numeric: NumericReport
    stats: CorrelationStats
    padded_shape: tuple = (0, 0, 0)


@dataclasses.dataclass
class CorrelationFailure:
    code: str
    message: str
    stats: CorrelationStats


@dataclasses.dataclass
class CorrelationEstimate:
    padded_shape: tuple
    padded_cells: int
    working_bytes: int


CorrelationOutcome = Union[CorrelationResult, CorrelationFailure]


class OperationControl:
    """Stop flag and deadline (runtime::OperationControl); polled between device phases."""

    def __init__(self, deadline_ns: int = 0):
        self._word = ctypes.c_uint32(0)
        self.deadline_ns = int(deadline_ns)

    def request_stop(self):
        self._word.value = 1

    def as_c(self) -> _lib.Control:
        return _lib.Control(ctypes.pointer(self._word), self.deadline_ns)

    def poll(self) -> Optional[str]:
        """The stop cause as the reference's code, or None (OperationControl::poll)."""
        if self._word.value:
            return "OPERATION_CANCELLED"
        if self.deadline_ns and time.monotonic_ns() >= self.deadline_ns:
            return "DEADLINE_EXCEEDED"
        return None


class Context:
    """A device context: stream, memory arena and the launch counter."""

    def __init__(self, device: int = 0, max_device_bytes: int = 0):
        handle = ctypes.c_void_p()
        check(lib().spk_context_create(device, max_device_bytes, ctypes.byref(handle)), "spk_context_create")
        self.handle = handle
        self.device = device

    def close(self):
        if self.handle:
            lib().spk_context_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def launches(self) -> int:
        return int(lib().spk_context_launches(self.handle))


_default: Optional[Context] = None


def default_context() -> Context:
    global _default
    if _default is None:
        _default = Context(0)
    return _default


def _spec_c(spec: CorrelationSpec) -> _lib.CorrelationSpec:
    c = _lib.CorrelationSpec()
    for a in range(3):
        c.environment_shape[a] = int(spec.environment_shape[a])
        c.kernel_shape[a] = int(spec.kernel_shape[a])
        c.environment_first[a] = int(spec.environment_first[a])
        c.kernel_first[a] = int(spec.kernel_first[a])
    return c


def estimate_correlation(spec: CorrelationSpec, precision: int = FP64) -> Union[CorrelationEstimate, CorrelationFailure]:
    out = _lib.CorrelationEstimateC()
    status = lib().spk_estimate_correlation(ctypes.byref(_spec_c(spec)), precision, ctypes.byref(out))
    if status:
        code = _lib.status_code(status)
        return CorrelationFailure(code, _MESSAGES.get(code, code), CorrelationStats())
    return CorrelationEstimate(tuple(out.padded_shape), out.padded_cells, out.working_bytes)


def _field_failure(es, ks, env, ker, control=None) -> Optional[CorrelationFailure]:
    """The reference's first checks, in its order (correlation.cpp:263-312):
    interruption, extents, then cell counts.  The library cannot see the cell
    counts, so a bad field fails here, before any device work; an
    interruption still wins over it, as in the reference.  Valid fields go to
    the library, which polls the control itself."""
    for code, bad in (("CORRELATION_SHAPE_OVERFLOW", min(es + ks) <= 0),
                      ("CORRELATION_INVALID_FIELD", env.size != int(np.prod(es, dtype=np.int64)) or
                       ker.size != int(np.prod(ks, dtype=np.int64)))):
        if bad:
            cause = control.poll() if control is not None else None
            code = cause or code
            return CorrelationFailure(code, _MESSAGES[code], CorrelationStats())
    return None


def _message(context) -> str:
    """The reference's message for the failing site (spk_context_message)."""
    f = lib().spk_context_message
    f.restype = ctypes.c_char_p
    f.argtypes = [ctypes.c_void_p]
    raw = f(context.handle)
    return raw.decode() if raw else ""


def _correlate(name, spec, environment, kernel, limits, control, precision, context, env_dtype):
    limits = limits or CorrelationLimits()
    es = [int(v) for v in spec.environment_shape]
    ks = [int(v) for v in spec.kernel_shape]
    env = np.ascontiguousarray(environment, dtype=env_dtype).reshape(-1)
    ker = np.ascontiguousarray(kernel, dtype=np.uint8).reshape(-1)
    bad = _field_failure(es, ks, env, ker, control)
    if bad is not None:
        return bad
    context = context or default_context()
    count = int(np.prod([e + k - 1 for e, k in zip(es, ks)], dtype=np.int64))
    out = np.empty(max(count, 1), np.float64)
    res = _lib.CorrelationResultC()
    lim = _lib.CorrelationLimits(limits.max_working_bytes, limits.reserved_bytes, limits.max_padded_cells,
                                 limits.max_direct_terms)
    ctl = control.as_c() if control is not None else None
    status = getattr(lib(), name)(context.handle, ctypes.byref(_spec_c(spec)), env.ctypes.data_as(ctypes.c_void_p),
                                  ker.ctypes.data_as(ctypes.c_void_p), ctypes.byref(lim),
                                  ctypes.byref(ctl) if ctl is not None else None, precision,
                                  out.ctypes.data_as(ctypes.c_void_p), out.size, ctypes.byref(res))
    stats = CorrelationStats(res.padded_cells, res.working_bytes_peak, res.direct_terms)
    if status:
        code = _lib.status_code(status)
        if code in ("CUDA_RUNTIME_ERROR", "SPK_INVALID_ARGUMENT"):
            raise SpkError(status, code, name)
        return CorrelationFailure(code, _message(context) or _MESSAGES.get(code, code), stats)
    return CorrelationResult(tuple(res.translation_first), tuple(res.shape), out[:count],
                             NumericReport(res.max_integer_residual, res.mass_residual, res.max_probe_error), stats,
                             tuple(res.padded_shape))


def correlate_binary(spec: CorrelationSpec, environment, kernel, limits: Optional[CorrelationLimits] = None,
                     control: Optional[OperationControl] = None, precision: int = FP32,
                     context: Optional[Context] = None) -> CorrelationOutcome:
    """GPU compute::correlate_binary_cpu: full-range overlap counts (rounded, checked)."""
    return _correlate("spk_correlate_binary", spec, environment, kernel, limits, control, precision, context,
                      np.uint8)


def correlate_binary_mask(spec: CorrelationSpec, environment, kernel, box_first: Sequence[int],
                          box_shape: Sequence[int], select: int = MASK_ZERO,
                          limits: Optional[CorrelationLimits] = None, control: Optional[OperationControl] = None,
                          precision: int = FP32, context: Optional[Context] = None,
                          capacity: Optional[int] = None) -> Union[MaskResult, CorrelationFailure]:
    """The binary correlation thresholded on the device: one byte per
    translation of the box instead of the full-range counts.  The gap-fill
    free mask (gap_fill.cpp:404-420) is the legal box with MASK_ZERO; the
    blocked offsets (gap_fill.cpp:443-446) and no-fit maps
    (slab_lattice.cpp:688-691) are the full range with MASK_NONZERO."""
    limits = limits or CorrelationLimits()
    es = [int(v) for v in spec.environment_shape]
    ks = [int(v) for v in spec.kernel_shape]
    env = np.ascontiguousarray(environment, dtype=np.uint8).reshape(-1)
    ker = np.ascontiguousarray(kernel, dtype=np.uint8).reshape(-1)
    bad = _field_failure(es, ks, env, ker, control)
    if bad is not None:
        return bad
    context = context or default_context()
    bf = (ctypes.c_int64 * 3)(*[int(v) for v in box_first])
    bs = (ctypes.c_uint32 * 3)(*[int(v) for v in box_shape])
    count = int(np.prod([int(v) for v in box_shape], dtype=np.int64))
    mask = np.zeros(max(count, 1), np.uint8)
    cap = count if capacity is None else int(capacity)
    res = _lib.CorrelationResultC()
    lim = _lib.CorrelationLimits(limits.max_working_bytes, limits.reserved_bytes, limits.max_padded_cells,
                                 limits.max_direct_terms)
    ctl = control.as_c() if control is not None else None
    status = lib().spk_correlate_binary_mask(
        context.handle, ctypes.byref(_spec_c(spec)), env.ctypes.data_as(ctypes.c_void_p),
        ker.ctypes.data_as(ctypes.c_void_p), ctypes.byref(lim), ctypes.byref(ctl) if ctl is not None else None,
        precision, bf, bs, select, mask.ctypes.data_as(ctypes.c_void_p), cap, ctypes.byref(res))
    stats = CorrelationStats(res.padded_cells, res.working_bytes_peak, res.direct_terms)
    if status:
        code = _lib.status_code(status)
        if code in ("CUDA_RUNTIME_ERROR", "SPK_INVALID_ARGUMENT"):
            raise SpkError(status, code, "spk_correlate_binary_mask")
        return CorrelationFailure(code, _MESSAGES.get(code, code), stats)
    return MaskResult(tuple(res.translation_first), tuple(res.shape), tuple(int(v) for v in box_first),
                      tuple(int(v) for v in box_shape), mask[:count],
                      NumericReport(res.max_integer_residual, res.mass_residual, res.max_probe_error), stats,
                      tuple(res.padded_shape))


def correlate_proximity(spec: CorrelationSpec, environment, kernel, limits: Optional[CorrelationLimits] = None,
                        control: Optional[OperationControl] = None, precision: int = FP64,
                        context: Optional[Context] = None) -> CorrelationOutcome:
    """GPU compute::correlate_proximity_cpu: full-range real correlation (checked)."""
    return _correlate("spk_correlate_proximity", spec, environment, kernel, limits, control, precision, context,
                      np.float64)


def build_proximity(shape: Sequence[int], occupied, context: Optional[Context] = None) -> Optional[np.ndarray]:
    """GPU solver::detail::build_proximity; None where the reference rejects the shape."""
    context = context or default_context()
    s = np.array(shape, np.uint32)
    occ = np.ascontiguousarray(occupied, dtype=np.uint8).reshape(-1)
    out = np.empty(occ.size, np.float64)
    status = lib().spk_build_proximity(context.handle, s.ctypes.data_as(ctypes.c_void_p),
                                       occ.ctypes.data_as(ctypes.c_void_p), out.ctypes.data_as(ctypes.c_void_p))
    if status == 21:
        return None
    check(status, "spk_build_proximity")
    return out


STATIC_PROXIMITY_MAX_AXIS = 64


def build_proximity_static(shape: Sequence[int], occupied_device_ptr: int, values_device_ptr: int,
                           stream: int = 0) -> None:
    """Allocation-free build_proximity for callers that cannot allocate device
    memory (no context, no cudaMalloc/cudaFree): `occupied_device_ptr` (u8)
    and `values_device_ptr` (f64) are caller-owned device addresses, `stream`
    a cudaStream_t handle (0 = default stream).  The scratch is one static
    device array shared by every call: fields larger than 64 cells on any axis
    raise SPK_SCRATCH_LIMIT, the first call on a device sets the array up and
    must come before any stream capture, and overlapping calls race."""
    s = np.array(shape, np.uint32)
    status = lib().spk_build_proximity_static(ctypes.c_void_p(stream or None), s.ctypes.data_as(ctypes.c_void_p),
                                              ctypes.c_void_p(occupied_device_ptr),
                                              ctypes.c_void_p(values_device_ptr))
    check(status, "spk_build_proximity_static")
