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

A ``WorkloadSpec`` holds only bytes and numbers (numpy, no library), so the
reference's own build can be driven with exactly the same inputs; ``Workload``
adds the accepted meshes and the catalog canonicalised by this library.
"""

from __future__ import annotations

import dataclasses
from typing import Optional, Union

import numpy as np

from . import synthetic
from .assets import AcceptedMesh, accept_stl


@dataclasses.dataclass
class WorkloadSpec:
    name: str
    object_stl: bytes
    container_box: Optional[tuple]  # box dimensions (mm), or None for the container STL
    container_stl: bytes
    origin: tuple
    pitch: float
    catalog_kind: str  # "cube" (24 axis rotations) or "hopf" (seeded SO(3) sample)
    catalog_count: int = 24
    catalog_seed: int = 0
    pair_clearance: float = 0.0
    wall_clearance: float = 0.0

    def raw_quaternions(self) -> Optional[np.ndarray]:
        """The Hopf-grid sample before canonicalisation; None for the cube catalog."""
        if self.catalog_kind != "hopf":
            return None
        from .geometry import hopf_quaternions

        return hopf_quaternions(self.catalog_count, self.catalog_seed)


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


def box64_cuboid_cube24_spec() -> WorkloadSpec:
    return WorkloadSpec("box64_cuboid_cube24", synthetic.cuboid_stl((10.0, 14.0, 20.0)), (64.0, 64.0, 64.0), b"",
                        (0.0, 0.0, 0.0), 1.0, "cube")


def box63_blob_hopf96_spec(seed: int = 1) -> WorkloadSpec:
    stl = synthetic.blob_stl(seed, level=4, base_mesh="icosahedron", radius_range=(6.0, 12.0))
    return WorkloadSpec("box63_blob_hopf96", stl, (63.0, 63.0, 63.0), b"", (0.0, 0.0, 0.0), 0.5, "hopf", 96, seed)


def rounded256_blob_hopf512_spec(seed: int = 2, orientations: int = 512) -> WorkloadSpec:
    container_stl = synthetic.rounded_box_stl((126.75, 126.75, 126.75), exponent=6.0, level=5,
                                              base_mesh="icosahedron")
    lo, hi = accept_stl(container_stl, role="container").bounds
    pitch = float((hi - lo).max()) / 253.5  # ceil(extent / pitch) = 254 -> 256 cells with the halo
    stl = synthetic.blob_stl(seed, level=5, base_mesh="octahedron", radius_range=(6.0, 12.0))
    return WorkloadSpec("rounded256_blob_hopf512", stl, None, container_stl, (0.0, 0.0, 0.0), pitch, "hopf",
                        orientations, seed)


def build(spec: WorkloadSpec) -> Workload:
    """Accepted meshes and this library's canonical catalog for a spec."""
    from .geometry import cube_catalog, custom_catalog

    catalog = cube_catalog() if spec.catalog_kind == "cube" else custom_catalog(spec.raw_quaternions())
    container = tuple(spec.container_box) if spec.container_box is not None else \
        accept_stl(spec.container_stl, role="container")
    return Workload(spec.name, accept_stl(spec.object_stl), container, spec.origin, spec.pitch, catalog,
                    spec.pair_clearance, spec.wall_clearance, object_stl=spec.object_stl,
                    container_stl=spec.container_stl)


def box64_cuboid_cube24() -> Workload:
    return build(box64_cuboid_cube24_spec())


def box63_blob_hopf96(seed: int = 1) -> Workload:
    return build(box63_blob_hopf96_spec(seed))


def rounded256_blob_hopf512(seed: int = 2, orientations: int = 512) -> Workload:
    return build(rounded256_blob_hopf512_spec(seed, orientations))


SPECS = {
    "box64_cuboid_cube24": box64_cuboid_cube24_spec,
    "box63_blob_hopf96": box63_blob_hopf96_spec,
    "rounded256_blob_hopf512": rounded256_blob_hopf512_spec,
}

WORKLOADS = {
    "box64_cuboid_cube24": box64_cuboid_cube24,
    "box63_blob_hopf96": box63_blob_hopf96,
    "rounded256_blob_hopf512": rounded256_blob_hopf512,
}
