"""Host mirror of the spectral page of the reference's build_spectral_pipeline.

Reference: engine/pack_solver/src/spectral_pipeline.hpp:26-51 (RankedCandidate,
CandidatePageQuery) and spectral_pipeline.cpp:1618-1857 (legal translations,
score, 32-entry page after an exclusive cursor, exact recount).
"""

from __future__ import annotations

import ctypes
import dataclasses
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from .compute import Context, default_context

PAGE_SIZE = 32


class CandidateC(ctypes.Structure):
    _fields_ = [("translation", ctypes.c_int64 * 3), ("score", ctypes.c_double),
                ("direct_zero_overlap", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("orientation_index", ctypes.c_uint64), ("binary_overlap", ctypes.c_double)]


class PageQueryC(ctypes.Structure):
    _fields_ = [("orientation_index", ctypes.c_uint64), ("has_cursor", ctypes.c_int32), ("mode", ctypes.c_int32),
                ("exclusive_cursor", CandidateC)]


class PageSceneC(ctypes.Structure):
    _fields_ = [("environment_first", ctypes.c_int64 * 3), ("environment_shape", ctypes.c_uint32 * 3),
                ("lattice_origin_mm", ctypes.c_double * 3), ("lattice_pitch_mm", ctypes.c_double),
                ("container_min_z_mm", ctypes.c_double), ("container_height_mm", ctypes.c_double)]


class PageKernelC(ctypes.Structure):
    _fields_ = [("first", ctypes.c_int64 * 3), ("shape", ctypes.c_uint32 * 3), ("object_max_z_mm", ctypes.c_double)]


class PageReportC(ctypes.Structure):
    _fields_ = [("max_integer_residual", ctypes.c_double), ("max_score_error", ctypes.c_double),
                ("rescored", ctypes.c_uint64), ("certified", ctypes.c_int32), ("threshold_pass", ctypes.c_int32)]


# One CandidateC as a numpy record: pages come back as one array and are
# converted column by column (a field read per ctypes element costs about
# twenty times as much).
CANDIDATE_DTYPE = np.dtype({"names": ["translation", "score", "direct_zero_overlap", "orientation_index",
                                      "binary_overlap"],
                            "formats": [("<i8", 3), "<f8", "<i4", "<u8", "<f8"],
                            "offsets": [CandidateC.translation.offset, CandidateC.score.offset,
                                        CandidateC.direct_zero_overlap.offset, CandidateC.orientation_index.offset,
                                        CandidateC.binary_overlap.offset],
                            "itemsize": ctypes.sizeof(CandidateC)})


# Slots and a field hash instead of frozen=True: a frozen dataclass sets each
# field through object.__setattr__, which made building a step's pages (up
# to 1,024 candidates) cost milliseconds of host time.
@dataclasses.dataclass(slots=True, unsafe_hash=True)
class RankedCandidate:
    translation: tuple
    score: float
    direct_zero_overlap: bool
    orientation_index: int
    binary_overlap: float

    def to_c(self) -> CandidateC:
        c = CandidateC()
        for a in range(3):
            c.translation[a] = int(self.translation[a])
        c.score = self.score
        c.direct_zero_overlap = int(self.direct_zero_overlap)
        c.orientation_index = int(self.orientation_index)
        c.binary_overlap = self.binary_overlap
        return c

    @staticmethod
    def from_c(c) -> "RankedCandidate":
        return RankedCandidate(tuple(int(v) for v in c.translation), float(c.score), bool(c.direct_zero_overlap),
                               int(c.orientation_index), float(c.binary_overlap))


def candidates_from_c(array, counts: Sequence[int], stride: int) -> List[List[RankedCandidate]]:
    """Pages out of a CandidateC array: page i is array[i * stride : i * stride
    + counts[i]], with the values RankedCandidate.from_c gives."""
    rec = np.frombuffer(array, dtype=CANDIDATE_DTYPE)
    translation = list(map(tuple, rec["translation"].tolist()))
    score = rec["score"].tolist()
    direct_zero = (rec["direct_zero_overlap"] != 0).tolist()
    orientation = rec["orientation_index"].tolist()
    overlap = rec["binary_overlap"].tolist()
    out = []
    for i, n in enumerate(counts):
        first = i * stride
        out.append([RankedCandidate(translation[j], score[j], direct_zero[j], orientation[j], overlap[j])
                    for j in range(first, first + int(n))])
    return out


@dataclasses.dataclass
class PageScene:
    environment_first: Sequence[int]
    environment_shape: Sequence[int]
    lattice_origin_mm: Sequence[float]
    lattice_pitch_mm: float
    container_min_z_mm: float
    container_height_mm: float


def _declare(lib):
    if getattr(lib, "_page_declared", False):
        return
    P = ctypes.c_void_p
    lib.spk_spectral_page.argtypes = [P, ctypes.POINTER(PageSceneC), P, ctypes.POINTER(PageKernelC), P,
                                      ctypes.POINTER(PageQueryC), ctypes.POINTER(CandidateC),
                                      ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(PageReportC)]
    lib._page_declared = True


def spectral_page(scene: PageScene, occupancy, kernel_first, kernel_shape, kernel_cells, object_max_z_mm: float,
                  orientation_index: int = 0, exclusive_cursor: Optional[RankedCandidate] = None,
                  context: Optional[Context] = None, report: Optional[dict] = None) -> List[RankedCandidate]:
    """One ordinary page (up to 32 candidates) for an oriented kernel over a layout."""
    lib = _lib.lib()
    _declare(lib)
    context = context or default_context()
    sc = PageSceneC()
    for a in range(3):
        sc.environment_first[a] = int(scene.environment_first[a])
        sc.environment_shape[a] = int(scene.environment_shape[a])
        sc.lattice_origin_mm[a] = float(scene.lattice_origin_mm[a])
    sc.lattice_pitch_mm = scene.lattice_pitch_mm
    sc.container_min_z_mm = scene.container_min_z_mm
    sc.container_height_mm = scene.container_height_mm
    kc = PageKernelC()
    for a in range(3):
        kc.first[a] = int(kernel_first[a])
        kc.shape[a] = int(kernel_shape[a])
    kc.object_max_z_mm = object_max_z_mm
    q = PageQueryC()
    q.orientation_index = orientation_index
    q.mode = 0
    if exclusive_cursor is not None:
        q.has_cursor = 1
        q.exclusive_cursor = exclusive_cursor.to_c()
    occ = np.ascontiguousarray(occupancy, dtype=np.uint8).reshape(-1)
    ker = np.ascontiguousarray(kernel_cells, dtype=np.uint8).reshape(-1)
    page = (CandidateC * PAGE_SIZE)()
    count = ctypes.c_uint32()
    rep = PageReportC()
    status = lib.spk_spectral_page(context.handle, ctypes.byref(sc), occ.ctypes.data_as(ctypes.c_void_p),
                                   ctypes.byref(kc), ker.ctypes.data_as(ctypes.c_void_p), ctypes.byref(q), page,
                                   ctypes.byref(count), ctypes.byref(rep))
    if report is not None:
        report.update(max_integer_residual=rep.max_integer_residual, max_score_error=rep.max_score_error,
                      rescored=rep.rescored, certified=bool(rep.certified), threshold_pass=bool(rep.threshold_pass))
    _lib.check(status, "spk_spectral_page")
    return candidates_from_c(page, [count.value], PAGE_SIZE)[0]
