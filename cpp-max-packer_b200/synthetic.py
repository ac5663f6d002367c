"""Seeded synthetic packing inputs, written as binary STL bytes.

The reference measures on user STL assets; the workloads here are seeded
stand-ins with the shapes named for the spectral placement benchmarks:

* ``cuboid_stl``: an axis-aligned cuboid as the 12-triangle binary STL a CAD
  exporter writes (8 corners, two triangles per face, outward winding).
* ``blob_stl``: a star-convex blob, radius ``base * (1 + sum c_lm Y_lm)`` over
  real spherical harmonics of degree 1..6 with seeded N(0, sigma) coefficients,
  meshed by radially displacing a subdivided octahedron or icosahedron.
* ``rounded_box_stl``: a superquadric ``|x/a|^p + |y/b|^p + |z/c|^p = 1``
  (a rounded box) meshed the same way, used as a closed STL container.

Vertices are rounded to float32 exactly as a binary STL stores them; the
engine's import step (anchoring and vertex welding, reference
engine/pack_geometry/src/import.cpp:509-660) happens in ``assets.accept_stl``.
"""

from __future__ import annotations

import math
import struct

import numpy as np

__all__ = [
    "cuboid_stl",
    "blob_stl",
    "rounded_box_stl",
    "sphere_mesh",
    "stl_bytes",
]


def stl_bytes(vertices: np.ndarray, triangles: np.ndarray) -> bytes:
    """Binary STL of an indexed mesh; normals are written as zero vectors."""
    v = np.asarray(vertices, dtype=np.float32)
    t = np.asarray(triangles, dtype=np.int64)
    records = np.zeros(len(t), dtype=[("n", "<f4", 3), ("v", "<f4", 9), ("a", "<u2")])
    records["v"] = v[t].reshape(len(t), 9)
    return b"spectrapack-b200 synthetic".ljust(80, b"\0") + struct.pack("<I", len(t)) + records.tobytes()


def cuboid_stl(size=(10.0, 14.0, 20.0)) -> bytes:
    sx, sy, sz = (float(s) for s in size)
    corners = np.array([[x, y, z] for z in (0.0, sz) for y in (0.0, sy) for x in (0.0, sx)])
    # Corner index = x + 2y + 4z (0/1 per axis).
    faces = [
        (0, 2, 3), (0, 3, 1),  # z = 0, normal -z
        (4, 5, 7), (4, 7, 6),  # z = sz, normal +z
        (0, 1, 5), (0, 5, 4),  # y = 0, normal -y
        (2, 6, 7), (2, 7, 3),  # y = sy, normal +y
        (0, 4, 6), (0, 6, 2),  # x = 0, normal -x
        (1, 3, 7), (1, 7, 5),  # x = sx, normal +x
    ]
    return stl_bytes(corners, np.array(faces))


def _subdivided(base: str, level: int):
    if base == "octahedron":
        verts = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
        faces = [(0, 2, 4), (2, 1, 4), (1, 3, 4), (3, 0, 4), (2, 0, 5), (1, 2, 5), (3, 1, 5), (0, 3, 5)]
    else:
        p = (1 + 5 ** 0.5) / 2
        verts = [(-1, p, 0), (1, p, 0), (-1, -p, 0), (1, -p, 0), (0, -1, p), (0, 1, p),
                 (0, -1, -p), (0, 1, -p), (p, 0, -1), (p, 0, 1), (-p, 0, -1), (-p, 0, 1)]
        faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
                 (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
                 (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    verts = [np.array(v, dtype=np.float64) / np.linalg.norm(v) for v in verts]
    for _ in range(level):
        cache: dict = {}
        new_faces = []

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            new_faces += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = new_faces
    return np.array(verts), np.array(faces, dtype=np.int64)


def sphere_mesh(level: int, base: str = "octahedron"):
    """Unit-sphere triangulation: directions (V,3) and outward triangles (F,3)."""
    return _subdivided(base, level)


def _real_sph_harm(l: int, m: int, theta: np.ndarray, phi: np.ndarray) -> np.ndarray:
    """Real spherical harmonic Y_lm (unnormalised Legendre form; scale is absorbed by the seeded coefficients)."""
    from scipy.special import lpmv

    am = abs(m)
    norm = math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(l - am) / math.factorial(l + am))
    leg = lpmv(am, l, np.cos(theta))
    if m > 0:
        return math.sqrt(2) * norm * leg * np.cos(am * phi)
    if m < 0:
        return math.sqrt(2) * norm * leg * np.sin(am * phi)
    return norm * leg


def blob_stl(seed: int, level: int = 4, base_mesh: str = "icosahedron", radius_range=(6.0, 12.0),
             degree: int = 6, sigma: float = 0.15) -> bytes:
    """Seeded star-convex blob; level 4 icosahedron = 5,120 triangles, level 5 octahedron = 8,192."""
    rng = np.random.default_rng(seed)
    base = rng.uniform(*radius_range)
    dirs, faces = sphere_mesh(level, base_mesh)
    theta = np.arccos(np.clip(dirs[:, 2], -1, 1))
    phi = np.arctan2(dirs[:, 1], dirs[:, 0])
    field = np.zeros(len(dirs))
    for l in range(1, degree + 1):
        for m in range(-l, l + 1):
            field += rng.normal(0.0, sigma) / l * _real_sph_harm(l, m, theta, phi)
    # Keep the surface star-convex and away from the centre.
    low = field.min()
    if low < -0.6:
        field *= 0.6 / -low
    radius = base * (1.0 + field)
    return stl_bytes(dirs * radius[:, None], faces)


def rounded_box_stl(half_extent=(126.75, 126.75, 126.75), exponent: float = 6.0, level: int = 6,
                    base_mesh: str = "octahedron") -> bytes:
    """Superquadric rounded box centred at the origin (level 6 octahedron = 32,768 triangles)."""
    dirs, faces = sphere_mesh(level, base_mesh)
    a = np.asarray(half_extent, dtype=np.float64)
    s = (np.abs(dirs / a) ** exponent).sum(axis=1) ** (-1.0 / exponent)
    return stl_bytes(dirs * s[:, None], faces)
