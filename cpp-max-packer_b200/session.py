"""A device-resident placement session: the B200 counterpart of the
reference's SpectralWorkspace plus its greedy placement loop.

Reference: engine/pack_solver/src/spectral_pipeline.hpp:67-99 (workspace and
build_spectral_pipeline pages) and engine/pack_solver/src/spectral.cpp:
1460-1591 (run_trial: page merge by rank_less, direct-zero gate, place at
origin + pitch * t).  Native validation stays with the caller, who can hand
it to the greedy loops as a validator (the reference's try_pose gate,
spectral.cpp:1289-1430).
"""

from __future__ import annotations

import ctypes
import dataclasses
from typing import List, Optional, Sequence, Union

import numpy as np

from . import _lib
from .assets import AcceptedMesh
from .compute import Context, default_context
from .geometry import MeshC, _lib_ready
from .pipeline import PAGE_SIZE, CandidateC, PageQueryC, PageReportC, RankedCandidate, candidates_from_c

P = ctypes.c_void_p
POSE_ACCEPTED, POSE_REJECTED = 0, 1
# int (*)(void* user, uint64 orientation, const int64 t[3], const double pose_mm[3], const double q[4])
VALIDATE_FN = ctypes.CFUNCTYPE(ctypes.c_int, P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int64),
                               ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double))


class SessionDescC(ctypes.Structure):
    _fields_ = [("object", MeshC), ("container_is_box", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("box_mm", ctypes.c_double * 3), ("container", MeshC), ("pair_clearance_mm", ctypes.c_double),
                ("wall_clearance_mm", ctypes.c_double), ("lattice_origin_mm", ctypes.c_double * 3),
                ("lattice_pitch_mm", ctypes.c_double), ("orientations_xyzw", P),
                ("orientation_count", ctypes.c_uint64)]


class SessionInfoC(ctypes.Structure):
    _fields_ = [("environment_first", ctypes.c_int64 * 3), ("environment_shape", ctypes.c_uint32 * 3),
                ("fft_shape", ctypes.c_uint32 * 3), ("copies", ctypes.c_uint64), ("orientations", ctypes.c_uint64),
                ("container_min_z_mm", ctypes.c_double), ("container_height_mm", ctypes.c_double)]


def _declare(lib):
    if getattr(lib, "_session_declared", False):
        return
    lib.spk_session_open.argtypes = [P, ctypes.POINTER(SessionDescC), ctypes.POINTER(SessionInfoC)]
    lib.spk_session_close.argtypes = [P]
    lib.spk_session_info_get.argtypes = [P, ctypes.POINTER(SessionInfoC)]
    lib.spk_session_place.argtypes = [P, ctypes.c_uint64, P]
    lib.spk_session_remove_last.argtypes = [P]
    lib.spk_session_pages.argtypes = [P, ctypes.c_uint64, ctypes.POINTER(PageQueryC), ctypes.POINTER(CandidateC),
                                      P, ctypes.POINTER(PageReportC)]
    lib.spk_session_greedy.argtypes = [P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64), P, P, P]
    lib.spk_session_field.argtypes = [P, ctypes.c_int, ctypes.c_uint64, P, P, P, ctypes.c_uint64]
    lib.spk_session_stats.argtypes = [P, P, ctypes.c_int]
    lib.spk_session_set_validator.argtypes = [P, VALIDATE_FN, P]
    lib.spk_session_validation_counts.argtypes = [P, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
    lib._session_declared = True


@dataclasses.dataclass
class Placement:
    orientation_index: int
    translation: tuple
    score: float


class Session:
    """Open with the accepted object mesh, a box (w, d, h) or container mesh,
    clearances, the lattice and a canonical orientation catalog."""

    def __init__(self, obj: AcceptedMesh, container: Union[Sequence[float], AcceptedMesh], lattice_origin_mm,
                 lattice_pitch_mm: float, catalog, pair_clearance_mm: float = 0.0, wall_clearance_mm: float = 0.0,
                 context: Optional[Context] = None):
        self.lib = _lib_ready()
        _declare(self.lib)
        self.context = context or default_context()
        self._keep = []
        d = SessionDescC()
        d.object = self._mesh(obj)
        if isinstance(container, AcceptedMesh):
            d.container_is_box = 0
            d.container = self._mesh(container)
        else:
            d.container_is_box = 1
            for a in range(3):
                d.box_mm[a] = float(container[a])
        d.pair_clearance_mm = pair_clearance_mm
        d.wall_clearance_mm = wall_clearance_mm
        for a in range(3):
            d.lattice_origin_mm[a] = float(lattice_origin_mm[a])
        d.lattice_pitch_mm = lattice_pitch_mm
        cat = np.ascontiguousarray(catalog, np.float64).reshape(-1, 4)
        self._keep.append(cat)
        d.orientations_xyzw = cat.ctypes.data
        d.orientation_count = len(cat)
        self.catalog = cat
        info = SessionInfoC()
        _lib.check(self.lib.spk_session_open(self.context.handle, ctypes.byref(d), ctypes.byref(info)),
                   "spk_session_open")
        self.origin = tuple(float(v) for v in lattice_origin_mm)
        self.pitch = lattice_pitch_mm
        self.environment_first = tuple(info.environment_first)
        self.environment_shape = tuple(info.environment_shape)
        self.fft_shape = tuple(info.fft_shape)
        self.placements: List[Placement] = []

    def _mesh(self, m: AcceptedMesh) -> MeshC:
        v = np.ascontiguousarray(m.vertices, np.float64)
        t = np.ascontiguousarray(m.triangles, np.uint32)
        self._keep += [v, t]
        return MeshC(v.ctypes.data, len(v), t.ctypes.data, len(t))

    def close(self):
        if self.context is not None and self.context.handle:
            self.lib.spk_session_close(self.context.handle)

    def place(self, orientation_index: int, translation) -> None:
        t = np.array(translation, np.int64)
        _lib.check(self.lib.spk_session_place(self.context.handle, orientation_index, t.ctypes.data),
                   "spk_session_place")
        self.placements.append(Placement(orientation_index, tuple(int(v) for v in t), float("nan")))

    def remove_last(self) -> None:
        _lib.check(self.lib.spk_session_remove_last(self.context.handle), "spk_session_remove_last")
        self.placements.pop()

    def pages(self, orientations, cursors=None, reports: Optional[list] = None,
              low_overlap: bool = False) -> List[List[RankedCandidate]]:
        """Ordinary pages, or with `low_overlap` the reference's low-overlap
        pages (every legal translation ranked by overlap count, then score)."""
        orientations = list(orientations)
        n = len(orientations)
        queries = (PageQueryC * n)()
        for i, o in enumerate(orientations):
            queries[i].orientation_index = o
            queries[i].mode = 1 if low_overlap else 0
            if cursors is not None and cursors[i] is not None:
                queries[i].has_cursor = 1
                queries[i].exclusive_cursor = cursors[i].to_c()
        pages = (CandidateC * (n * PAGE_SIZE))()
        counts = np.zeros(n, np.uint32)
        reps = (PageReportC * n)()
        _lib.check(self.lib.spk_session_pages(self.context.handle, n, queries, pages, counts.ctypes.data, reps),
                   "spk_session_pages")
        if reports is not None:
            reports.extend(dict(max_integer_residual=r.max_integer_residual, max_score_error=r.max_score_error,
                                rescored=r.rescored, certified=bool(r.certified),
                                threshold_pass=bool(r.threshold_pass)) for r in reps)
        return candidates_from_c(pages, counts.tolist(), PAGE_SIZE)

    def greedy(self, max_steps: int) -> List[Placement]:
        ori = np.zeros(max(max_steps, 1), np.uint64)
        t = np.zeros((max(max_steps, 1), 3), np.int64)
        scores = np.zeros(max(max_steps, 1), np.float64)
        placed = ctypes.c_uint64()
        _lib.check(self.lib.spk_session_greedy(self.context.handle, max_steps, ctypes.byref(placed), ori.ctypes.data,
                                               t.ctypes.data, scores.ctypes.data), "spk_session_greedy")
        out = [Placement(int(ori[i]), tuple(int(v) for v in t[i]), float(scores[i])) for i in range(placed.value)]
        self.placements += out
        return out

    def set_validator(self, validate) -> None:
        """`validate(orientation, translation, pose_mm, quaternion_xyzw)`
        returns True to accept a chosen pose, False to reject it (the greedy
        moves on to the next candidate); an exception stops the fill with
        SPECTRAL_VALIDATION_ABORTED.  None removes the validator."""
        if validate is None:
            self._validator = None
            _lib.check(self.lib.spk_session_set_validator(self.context.handle, VALIDATE_FN(), None),
                       "spk_session_set_validator")
            return

        def call(_user, orientation, t, pose, q):
            try:
                ok = validate(int(orientation), tuple(t[a] for a in range(3)), tuple(pose[a] for a in range(3)),
                              tuple(q[a] for a in range(4)))
            except Exception:  # noqa: BLE001 - reported to the library as an abort
                return 2
            return POSE_ACCEPTED if ok else POSE_REJECTED

        self._validator = VALIDATE_FN(call)
        _lib.check(self.lib.spk_session_set_validator(self.context.handle, self._validator, None),
                   "spk_session_set_validator")

    def validation_counts(self) -> tuple:
        """(poses validated, poses rejected) since the session opened."""
        v, r = ctypes.c_uint64(), ctypes.c_uint64()
        _lib.check(self.lib.spk_session_validation_counts(self.context.handle, ctypes.byref(v), ctypes.byref(r)),
                   "spk_session_validation_counts")
        return int(v.value), int(r.value)

    def stats(self, reset: bool = False) -> dict:
        out = np.zeros(4, np.uint64)
        _lib.check(self.lib.spk_session_stats(self.context.handle, out.ctypes.data, int(reset)), "spk_session_stats")
        return {"pages": int(out[0]), "threshold_passes": int(out[1]), "rescored": int(out[2]),
                "first_pass_certified": int(out[3])}

    def field(self, kind: str, orientation: int = 0) -> np.ndarray:
        code = {"container": 0, "occupancy": 1, "kernel": 2, "proximity": 3}[kind]
        first = np.zeros(3, np.int64)
        shape = np.zeros(3, np.uint32)
        _lib.check(self.lib.spk_session_field(self.context.handle, code, orientation, first.ctypes.data,
                                              shape.ctypes.data, None, 0), "spk_session_field")
        n = int(np.prod(shape.astype(np.int64)))
        out = np.zeros(n, np.float64 if code == 3 else np.uint8)
        _lib.check(self.lib.spk_session_field(self.context.handle, code, orientation, first.ctypes.data,
                                              shape.ctypes.data, out.ctypes.data, out.nbytes), "spk_session_field")
        self.last_window = (tuple(int(v) for v in first), tuple(int(v) for v in shape))
        return out


class JobC(ctypes.Structure):
    _fields_ = [("context", P), ("proposal", P), ("k", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
                ("max_steps", ctypes.c_uint64), ("orientations", P), ("translations", P), ("scores", P),
                ("placed", ctypes.c_uint64), ("fallbacks", ctypes.c_uint64), ("status", ctypes.c_int32),
                ("reserved2", ctypes.c_int32)]


def run_jobs(jobs) -> list:
    """Fills several sessions concurrently (spk_jobs_greedy).  `jobs` holds
    (session, proposal or None, k, max_steps) tuples, every session on its own
    context; returns (placements, fallback steps) per job, in order."""
    lib = _lib_ready()
    _declare(lib)
    if not getattr(lib, "_jobs_declared", False):
        lib.spk_jobs_greedy.argtypes = [ctypes.POINTER(JobC), ctypes.c_uint64]
        lib._jobs_declared = True
    arr = (JobC * len(jobs))()
    keep = []
    for i, (session, net, k, max_steps) in enumerate(jobs):
        n = max(int(max_steps), 1)
        ori = np.zeros(n, np.uint64)
        t = np.zeros((n, 3), np.int64)
        scores = np.zeros(n, np.float64)
        keep.append((ori, t, scores))
        arr[i].context = session.context.handle
        arr[i].proposal = net.handle if net is not None else None
        arr[i].k = int(k)
        arr[i].max_steps = int(max_steps)
        arr[i].orientations = ori.ctypes.data
        arr[i].translations = t.ctypes.data
        arr[i].scores = scores.ctypes.data
    _lib.check(lib.spk_jobs_greedy(arr, len(jobs)), "spk_jobs_greedy")
    out = []
    for i, (session, _, _, _) in enumerate(jobs):
        _lib.check(arr[i].status, f"spk_jobs_greedy job {i}")
        ori, t, scores = keep[i]
        placed = [Placement(int(ori[j]), tuple(int(v) for v in t[j]), float(scores[j]))
                  for j in range(arr[i].placed)]
        session.placements += placed
        out.append((placed, int(arr[i].fallbacks)))
    return out
