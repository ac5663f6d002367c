"""STL export of a placement sequence (spk_export_stl) against the reference's
record loop (pack_io's write_stl_stage, result_export.cpp:1034-1123, run in
the reference build with its own RigidTransform and the host's hypot): the
files must be byte-identical.

Poses: seeded general rotations of a blob, cardinal and general rotations of
a cuboid, and the poses of a GPU greedy fill (translation = origin + pitch *
cell, the reference's CopyPose expression at spectral.cpp:1571-1577).
Failures: a pose without a rigid transform and a buffer that is too small.
"""

import importlib

import numpy as np
import pytest

from conftest import package

pytestmark = pytest.mark.gpu
syn = importlib.import_module("cpp-max-packer_b200.synthetic")


def _rotations(rng, n):
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1)[:, None]
    q[q[:, 3] < 0] *= -1
    return q


@pytest.mark.parametrize("item,cardinal", [("blob", False), ("cuboid", True), ("cuboid", False)])
def test_stl_bytes_match_reference(gpu_ctx, oracle_ref, item, cardinal):
    assets, geometry = package("assets"), package("geometry")
    stl = syn.blob_stl(9, level=4, radius_range=(4.0, 9.0)) if item == "blob" else syn.cuboid_stl((7.0, 4.5, 3.25))
    mesh = assets.accept_stl(stl)
    ref_asset = oracle_ref.asset(stl)
    rng = np.random.default_rng(17 + int(cardinal))
    n = 60
    q = geometry.cube_catalog()[rng.integers(0, 24, size=n)] if cardinal else _rotations(rng, n)
    t = rng.uniform(-300.0, 300.0, size=(n, 3))
    got = geometry.export_stl(mesh, t, q, context=gpu_ctx)
    want = ref_asset.export_stl(t, q)
    assert len(got) == len(want) == 84 + 50 * len(mesh.triangles) * n
    assert got == want


def test_stl_of_a_fill_matches_reference(gpu_ctx, oracle_ref):
    geometry, session_mod, workloads = package("geometry"), package("session"), package("workloads")
    wl = workloads.rounded256_blob_hopf512(orientations=16)
    s = session_mod.Session(wl.obj, wl.container, wl.origin, wl.pitch, wl.catalog, context=gpu_ctx)
    placed = s.greedy(12)
    s.close()
    t = np.array([[wl.origin[a] + wl.pitch * p.translation[a] for a in range(3)] for p in placed])
    q = np.array([wl.catalog[p.orientation_index] for p in placed])
    got = geometry.export_stl(wl.obj, t, q, context=gpu_ctx)
    assert got == oracle_ref.asset(wl.object_stl).export_stl(t, q)


def test_stl_export_failures(gpu_ctx):
    assets, geometry, lib_mod = package("assets"), package("geometry"), package("_lib")
    mesh = assets.accept_stl(syn.cuboid_stl((2.0, 3.0, 4.0)))
    with pytest.raises(lib_mod.SpkError) as err:
        geometry.export_stl(mesh, [[0.0, 0.0, 0.0]], [[0.0, 0.0, 0.0, 0.0]], context=gpu_ctx)
    assert err.value.status == 15
    with pytest.raises(lib_mod.SpkError) as err:
        geometry.export_stl(mesh, [[1e39, 0.0, 0.0]], [[0.0, 0.0, 0.0, 1.0]], context=gpu_ctx)
    assert err.value.status == 15
