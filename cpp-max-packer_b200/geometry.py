"""Host mirror of the reference's conservative-field factories on the B200 path.

Reference interface (engine/pack_geometry/include/spectrapack/geometry/
conservative_fields.hpp:100-164): voxelize_object(geometry, lattice,
rotation), voxelize_container(container, window, clearance) and
voxelize_placed(geometry, window, pose, clearance) return CellFields (a
window plus X-fastest u8 cells) or a RepresentationFailure code.  The
functions here take the accepted local mesh directly and raise SpkError
with the reference's code on failure.
"""

from __future__ import annotations

import ctypes
import dataclasses
from typing import Optional, Sequence, Union

import numpy as np

from . import _lib
from .assets import AcceptedMesh
from .compute import Context, default_context

P = ctypes.c_void_p


class MeshC(ctypes.Structure):
    _fields_ = [("vertices", P), ("vertex_count", ctypes.c_uint64), ("triangles", P),
                ("triangle_count", ctypes.c_uint64)]


@dataclasses.dataclass
class CellField:
    first: tuple
    shape: tuple
    cells: np.ndarray  # X-fastest u8

    def dense(self) -> np.ndarray:
        return self.cells.reshape(self.shape[2], self.shape[1], self.shape[0])


def _mesh_c(mesh: AcceptedMesh):
    v = np.ascontiguousarray(mesh.vertices, np.float64)
    t = np.ascontiguousarray(mesh.triangles, np.uint32)
    return MeshC(v.ctypes.data, len(v), t.ctypes.data, len(t)), (v, t)


def _declare(lib):
    if getattr(lib, "_geometry_declared", False):
        return
    M = ctypes.POINTER(MeshC)
    lib.spk_voxelize_object.argtypes = [P, M, P, ctypes.c_double, P, P, P, P, ctypes.c_uint64]
    lib.spk_voxelize_container.argtypes = [P, P, M, P, ctypes.c_double, P, P, ctypes.c_double, P]
    lib.spk_voxelize_placed.argtypes = [P, M, P, ctypes.c_double, P, P, P, P, ctypes.c_double, P]
    lib.spk_oriented_bounds.argtypes = [M, P, P]
    lib.spk_posed_bounds.argtypes = [M, P, P, ctypes.c_uint64, P, P, P]
    lib.spk_export_stl.argtypes = [P, M, P, P, ctypes.c_uint64, P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]
    lib.spk_broad_phase.argtypes = [P, P, P, P, P, ctypes.c_uint64, ctypes.c_double, P, ctypes.c_uint64,
                                    ctypes.POINTER(ctypes.c_uint64)]
    lib.spk_environment_window.argtypes = [P, P, ctypes.c_double, P, P]
    lib.spk_cube_catalog.argtypes = [P]
    lib.spk_custom_catalog.argtypes = [P, ctypes.c_uint64, P, ctypes.POINTER(ctypes.c_uint64)]
    lib._geometry_declared = True


def _lib_ready():
    lib = _lib.lib()
    _declare(lib)
    return lib


def _arr(values, dtype):
    return np.ascontiguousarray(np.array(values, dtype=dtype))


def voxelize_object(mesh: AcceptedMesh, origin_mm: Sequence[float], pitch_mm: float, q_xyzw: Sequence[float],
                    context: Optional[Context] = None, capacity: int = 1 << 26) -> CellField:
    lib = _lib_ready()
    context = context or default_context()
    mc, keep = _mesh_c(mesh)
    first = np.zeros(3, np.int64)
    shape = np.zeros(3, np.uint32)
    o, q = _arr(origin_mm, np.float64), _arr(q_xyzw, np.float64)
    cells = np.zeros(capacity, np.uint8)
    status = lib.spk_voxelize_object(context.handle, ctypes.byref(mc), o.ctypes.data, pitch_mm, q.ctypes.data,
                                     first.ctypes.data, shape.ctypes.data, cells.ctypes.data, capacity)
    _lib.check(status, "spk_voxelize_object")
    n = int(np.prod(shape.astype(np.int64)))
    return CellField(tuple(int(v) for v in first), tuple(int(v) for v in shape), cells[:n].copy())


def voxelize_container(container: Union[Sequence[float], AcceptedMesh], origin_mm, pitch_mm, first, shape,
                       wall_clearance_mm: float = 0.0, context: Optional[Context] = None) -> CellField:
    """Box dimensions (width, depth, height) or a container mesh; 1 = blocked."""
    lib = _lib_ready()
    context = context or default_context()
    f, s = _arr(first, np.int64), _arr(shape, np.uint32)
    cells = np.zeros(int(np.prod(s.astype(np.int64))), np.uint8)
    o = _arr(origin_mm, np.float64)
    if isinstance(container, AcceptedMesh):
        mc, keep = _mesh_c(container)
        status = lib.spk_voxelize_container(context.handle, None, ctypes.byref(mc), o.ctypes.data, pitch_mm,
                                            f.ctypes.data, s.ctypes.data, wall_clearance_mm, cells.ctypes.data)
    else:
        box = _arr(container, np.float64)
        status = lib.spk_voxelize_container(context.handle, box.ctypes.data, None, o.ctypes.data, pitch_mm,
                                            f.ctypes.data, s.ctypes.data, wall_clearance_mm, cells.ctypes.data)
    _lib.check(status, "spk_voxelize_container")
    return CellField(tuple(int(v) for v in f), tuple(int(v) for v in s), cells)


def voxelize_placed(mesh: AcceptedMesh, origin_mm, pitch_mm, first, shape, translation_mm, q_xyzw,
                    pair_clearance_mm: float = 0.0, context: Optional[Context] = None) -> CellField:
    lib = _lib_ready()
    context = context or default_context()
    mc, keep = _mesh_c(mesh)
    f, s = _arr(first, np.int64), _arr(shape, np.uint32)
    cells = np.zeros(int(np.prod(s.astype(np.int64))), np.uint8)
    o, t, q = _arr(origin_mm, np.float64), _arr(translation_mm, np.float64), _arr(q_xyzw, np.float64)
    status = lib.spk_voxelize_placed(context.handle, ctypes.byref(mc), o.ctypes.data, pitch_mm, f.ctypes.data,
                                     s.ctypes.data, t.ctypes.data, q.ctypes.data, pair_clearance_mm,
                                     cells.ctypes.data)
    _lib.check(status, "spk_voxelize_placed")
    return CellField(tuple(int(v) for v in f), tuple(int(v) for v in s), cells)


def oriented_bounds(mesh: AcceptedMesh, q_xyzw) -> np.ndarray:
    lib = _lib_ready()
    mc, keep = _mesh_c(mesh)
    out = np.zeros(6, np.float64)
    q = _arr(q_xyzw, np.float64)
    _lib.check(lib.spk_oriented_bounds(ctypes.byref(mc), q.ctypes.data, out.ctypes.data), "spk_oriented_bounds")
    return out


def posed_bounds(mesh: AcceptedMesh, translations_mm, quaternions_xyzw):
    """validation_kernel::posed_bounds of each pose (validation_kernel.cpp:1000-1088):
    (min (n, 3), max (n, 3), finite (n,) bool)."""
    lib = _lib_ready()
    mc, keep = _mesh_c(mesh)
    t = _arr(translations_mm, np.float64).reshape(-1, 3)
    q = _arr(quaternions_xyzw, np.float64).reshape(-1, 4)
    n = len(t)
    lo, hi = np.zeros((n, 3), np.float64), np.zeros((n, 3), np.float64)
    finite = np.zeros(n, np.uint8)
    _lib.check(lib.spk_posed_bounds(ctypes.byref(mc), t.ctypes.data, q.ctypes.data, n, lo.ctypes.data,
                                    hi.ctypes.data, finite.ctypes.data), "spk_posed_bounds")
    return lo, hi, finite.astype(bool)


def broad_phase(bounds_min, bounds_max, finite, clearance_mm: float, proven=None,
                context: Optional[Context] = None, capacity: Optional[int] = None) -> np.ndarray:
    """The copy pairs the validator's outward-AABB test leaves unresolved
    (validation.cpp:404-418), (count, 2) uint32 rows (first, second) in its
    visiting order."""
    lib = _lib_ready()
    context = context or default_context()
    lo = _arr(bounds_min, np.float64).reshape(-1, 3)
    hi = _arr(bounds_max, np.float64).reshape(-1, 3)
    n = len(lo)
    fin = _arr(finite, np.uint8)
    prv = None if proven is None else _arr(proven, np.uint8)
    cap = n * (n - 1) // 2 if capacity is None else capacity
    out = np.zeros((max(cap, 1), 2), np.uint32)
    count = ctypes.c_uint64()
    _lib.check(lib.spk_broad_phase(context.handle, lo.ctypes.data, hi.ctypes.data, fin.ctypes.data,
                                   None if prv is None else prv.ctypes.data, n, clearance_mm, out.ctypes.data, cap,
                                   ctypes.byref(count)), "spk_broad_phase")
    return out[:count.value].copy()


def export_stl(mesh: AcceptedMesh, translations_mm, quaternions_xyzw, context: Optional[Context] = None,
               out: Optional[np.ndarray] = None):
    """The binary STL of the posed copies (pack_io's write_stl_stage,
    result_export.cpp:1034-1123), computed on the device: the file's bytes,
    or, with `out` (a uint8 array at least as large), the file's size after
    writing it there."""
    lib = _lib_ready()
    context = context or default_context()
    mc, keep = _mesh_c(mesh)
    t = _arr(translations_mm, np.float64).reshape(-1, 3)
    q = _arr(quaternions_xyzw, np.float64).reshape(-1, 4)
    size = 84 + 50 * len(mesh.triangles) * len(t)
    buffer = np.empty(size, np.uint8) if out is None else out
    got = ctypes.c_uint64()
    _lib.check(lib.spk_export_stl(context.handle, ctypes.byref(mc), t.ctypes.data, q.ctypes.data, len(t),
                                  buffer.ctypes.data, buffer.nbytes, ctypes.byref(got)), "spk_export_stl")
    return buffer[:got.value].tobytes() if out is None else int(got.value)


def environment_window(bounds_mm, origin_mm, pitch_mm):
    lib = _lib_ready()
    b, o = _arr(bounds_mm, np.float64), _arr(origin_mm, np.float64)
    first = np.zeros(3, np.int64)
    shape = np.zeros(3, np.uint32)
    _lib.check(lib.spk_environment_window(b.ctypes.data, o.ctypes.data, pitch_mm, first.ctypes.data,
                                          shape.ctypes.data), "spk_environment_window")
    return tuple(int(v) for v in first), tuple(int(v) for v in shape)


def cube_catalog() -> np.ndarray:
    lib = _lib_ready()
    out = np.zeros((24, 4), np.float64)
    _lib.check(lib.spk_cube_catalog(out.ctypes.data), "spk_cube_catalog")
    return out


def custom_catalog(quaternions) -> np.ndarray:
    lib = _lib_ready()
    q = np.ascontiguousarray(quaternions, np.float64).reshape(-1, 4)
    out = np.zeros_like(q)
    count = ctypes.c_uint64()
    _lib.check(lib.spk_custom_catalog(q.ctypes.data, len(q), out.ctypes.data, ctypes.byref(count)),
               "spk_custom_catalog")
    return out[: count.value].copy()


def hopf_quaternions(count: int, seed: int) -> np.ndarray:
    """Seeded uniform SO(3) sample: unit XYZW quaternions by Shoemake's
    subgroup algorithm, before canonicalisation (numpy only)."""
    rng = np.random.default_rng(seed)
    u1, u2, u3 = rng.random(count), rng.random(count), rng.random(count)
    return np.stack([np.sqrt(1 - u1) * np.sin(2 * np.pi * u2), np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
                     np.sqrt(u1) * np.sin(2 * np.pi * u3), np.sqrt(u1) * np.cos(2 * np.pi * u3)], axis=1)


def hopf_catalog(count: int, seed: int) -> np.ndarray:
    """hopf_quaternions made canonical and de-duplicated like a custom catalog."""
    return custom_catalog(hopf_quaternions(count, seed))
