"""The seeded spectral-placement workloads used by the bench, smoke check and tests.

Each workload is a seeded synthetic stand-in with the shapes, sizes and
orientation counts of the spectral placement benchmark configurations:

* ``box64_cuboid_cube24``: a 64 x 64 x 64 mm box at 1 mm (66^3 window with the
  one-cell halo), a 10 x 14 x 20 mm cuboid as a 12-triangle binary STL and the
  24 cube orientations.
* ``box63_blob_hopf96``: a 63 mm box at 0.5 mm (128^3 window), a star-convex
  spherical-harmonic blob (5,120 triangles, radius 6-12 mm) and 96 seeded
  uniform SO(3) orientations.
* ``rounded256_blob_hopf512``: a closed rounded-box container STL
  (superquadric, 20,480 triangles) whose window is 256^3 at 1 mm, the same blob
  generator meshed to 8,192 triangles, and 512 seeded SO(3) orientations.
"""

from __future__ import annotations

import dataclasses
from typing import Union

import numpy as np

from . import synthetic
from .assets import AcceptedMesh, accept_stl


@dataclasses.dataclass
class Workload:
    name: str
    obj: AcceptedMesh
    container: Union[tuple, AcceptedMesh]
    origin: tuple
    pitch: float
    catalog: np.ndarray
    pair_clearance: float = 0.0
    wall_clearance: float = 0.0
    object_stl: bytes = b""
    container_stl: bytes = b""


def _catalog_cube():
    from .geometry import cube_catalog

    return cube_catalog()


def _catalog_hopf(count, seed):
    from .geometry import hopf_catalog

    return hopf_catalog(count, seed)


def box64_cuboid_cube24() -> Workload:
    stl = synthetic.cuboid_stl((10.0, 14.0, 20.0))
    return Workload("box64_cuboid_cube24", accept_stl(stl), (64.0, 64.0, 64.0), (0.0, 0.0, 0.0), 1.0,
                    _catalog_cube(), object_stl=stl)


def box63_blob_hopf96(seed: int = 1) -> Workload:
    stl = synthetic.blob_stl(seed, level=4, base_mesh="icosahedron", radius_range=(6.0, 12.0))
    return Workload("box63_blob_hopf96", accept_stl(stl), (63.0, 63.0, 63.0), (0.0, 0.0, 0.0), 0.5,
                    _catalog_hopf(96, seed), object_stl=stl)


def rounded256_blob_hopf512(seed: int = 2, orientations: int = 512) -> Workload:
    container_stl = synthetic.rounded_box_stl((126.75, 126.75, 126.75), exponent=6.0, level=5,
                                              base_mesh="icosahedron")
    container = accept_stl(container_stl, role="container")
    lo, hi = container.bounds
    pitch = float((hi - lo).max()) / 253.5  # ceil(extent / pitch) = 254 -> 256 cells with the halo
    stl = synthetic.blob_stl(seed, level=5, base_mesh="octahedron", radius_range=(6.0, 12.0))
    return Workload("rounded256_blob_hopf512", accept_stl(stl), container, (0.0, 0.0, 0.0), pitch,
                    _catalog_hopf(orientations, seed), object_stl=stl, container_stl=container_stl)


WORKLOADS = {
    "box64_cuboid_cube24": box64_cuboid_cube24,
    "box63_blob_hopf96": box63_blob_hopf96,
    "rounded256_blob_hopf512": rounded256_blob_hopf512,
}
