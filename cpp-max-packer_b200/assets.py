"""Binary STL to an accepted local mesh, as the engine's import hands it over.

The reference engine accepts an STL through inspect_stl/accept_asset
(engine/pack_geometry/src/import.cpp:509-660) and the hot path only ever sees
AcceptedSolid::mesh(): welded vertices in a local frame.  The steps restated
here, for closed, outward-wound meshes (the synthetic inputs):

* the frame comes from the bounds of the parsed (float32) vertices; the anchor
  is the lower corner for a container and lo/2 + hi/2 for an object;
* exactly equal vertices merge in first-appearance order (-0 counts as +0);
* faces whose three vertices are collinear (exact test) and cyclic duplicates
  are dropped; unreferenced vertices are compacted away;
* local = scale * v - anchor, with -0 normalised to +0.
"""

from __future__ import annotations

import dataclasses
import struct
from fractions import Fraction

import numpy as np


@dataclasses.dataclass
class AcceptedMesh:
    vertices: np.ndarray   # (V, 3) float64, local frame
    triangles: np.ndarray  # (F, 3) uint32
    role: str              # "object" or "container"

    @property
    def bounds(self):
        return self.vertices.min(axis=0), self.vertices.max(axis=0)


def parse_binary_stl(data: bytes) -> np.ndarray:
    """(F, 3, 3) float64 triangle soup of a binary STL (float32 values)."""
    if len(data) < 84:
        raise ValueError("binary STL header is truncated")
    (count,) = struct.unpack_from("<I", data, 80)
    if len(data) != 84 + 50 * count or count == 0:
        raise ValueError("binary STL size does not match its triangle count")
    records = np.frombuffer(data, dtype=[("n", "<f4", 3), ("v", "<f4", 9), ("a", "<u2")], count=count, offset=84)
    return records["v"].astype(np.float64).reshape(count, 3, 3)


def _collinear(a, b, c) -> bool:
    u = [Fraction(b[i]) - Fraction(a[i]) for i in range(3)]
    v = [Fraction(c[i]) - Fraction(a[i]) for i in range(3)]
    return (u[1] * v[2] - u[2] * v[1] == 0 and u[2] * v[0] - u[0] * v[2] == 0 and u[0] * v[1] - u[1] * v[0] == 0)


def accept_stl(data: bytes, role: str = "object", scale: float = 1.0) -> AcceptedMesh:
    soup = parse_binary_stl(data)
    pts = soup.reshape(-1, 3)
    lo = pts.min(axis=0) * scale
    hi = pts.max(axis=0) * scale
    anchor = lo.copy() if role == "container" else lo / 2.0 + hi / 2.0
    anchor = np.where(anchor == 0.0, 0.0, anchor)
    pts = np.where(pts == 0.0, 0.0, pts)
    index: dict = {}
    unique = []
    remap = np.empty(len(pts), np.int64)
    for i, p in enumerate(map(tuple, pts)):
        at = index.get(p)
        if at is None:
            at = index[p] = len(unique)
            unique.append(p)
        remap[i] = at
    unique = np.array(unique, np.float64)
    faces = remap.reshape(-1, 3)
    # float filter, exact confirmation for nearly degenerate faces
    a, b, c = unique[faces[:, 0]], unique[faces[:, 1]], unique[faces[:, 2]]
    cross = np.cross(b - a, c - a)
    scale_term = np.abs(b - a).max(axis=1) * np.abs(c - a).max(axis=1)
    suspect = np.abs(cross).max(axis=1) <= 1e-12 * np.maximum(scale_term, 1e-300)
    kept = []
    seen = set()
    for f, face in enumerate(faces):
        if suspect[f] and _collinear(*unique[face]):
            continue
        t = tuple(int(v) for v in face)
        cyc = min(t, (t[1], t[2], t[0]), (t[2], t[0], t[1]))
        if cyc in seen:
            continue
        seen.add(cyc)
        kept.append(t)
    kept = np.array(kept, np.int64)
    referenced = np.zeros(len(unique), bool)
    referenced[kept.reshape(-1)] = True
    compact = np.cumsum(referenced) - 1
    local = scale * unique[referenced] - anchor
    local = np.where(local == 0.0, 0.0, local)
    return AcceptedMesh(np.ascontiguousarray(local), np.ascontiguousarray(compact[kept].astype(np.uint32)), role)
