"""Host-only geometry entry points against the reference's outputs (CPU)."""

import os

import numpy as np
import pytest

from conftest import ROOT, package

GOLD = np.load(os.path.join(ROOT, "tests", "golden", "fields.npz"))
CASES = ["cuboid", "cuboid_offset", "blob", "blob_fine"]


@pytest.mark.parametrize("name", CASES)
def test_accepted_mesh_matches_reference_import(name):
    assets = package("assets")
    mesh = assets.accept_stl(GOLD[f"{name}/stl"].tobytes())
    assert np.array_equal(mesh.vertices.view(np.uint64), GOLD[f"{name}/vertices"].view(np.uint64))
    assert np.array_equal(mesh.triangles, GOLD[f"{name}/triangles"])


def test_container_mesh_matches_reference_import():
    assets = package("assets")
    mesh = assets.accept_stl(GOLD["container/rounded/stl"].tobytes(), role="container")
    assert np.array_equal(mesh.vertices.view(np.uint64), GOLD["container/rounded/vertices"].view(np.uint64))
    assert np.array_equal(mesh.triangles, GOLD["container/rounded/triangles"])


def test_cube_catalog_matches_reference_order():
    geometry = package("geometry")
    assert np.array_equal(geometry.cube_catalog(), GOLD["cube_catalog"])


@pytest.mark.parametrize("name", CASES)
def test_oriented_bounds_bit_exact(name):
    assets, geometry = package("assets"), package("geometry")
    mesh = assets.accept_stl(GOLD[f"{name}/stl"].tobytes())
    for i, q in enumerate(GOLD[f"{name}/quaternions"]):
        got = geometry.oriented_bounds(mesh, q)
        assert np.array_equal(got.view(np.uint64), GOLD[f"{name}/bounds{i}"].view(np.uint64))


def test_custom_catalog_canonical_and_dedup():
    geometry = package("geometry")
    q = np.array([[0, 0, 0, -2.0], [0, 0, 0, 1.0], [0.5, 0.5, 0.5, 0.5], [-0.5, -0.5, -0.5, -0.5], [0, -1.0, 0, 0]])
    out = geometry.custom_catalog(q)
    assert out.tolist() == [[0, 0, 0, 1.0], [0.5, 0.5, 0.5, 0.5], [0, 1.0, 0, 0]]


def test_environment_window_halo():
    geometry = package("geometry")
    assert geometry.environment_window((0, 0, 0, 64, 64, 64), (0, 0, 0), 1.0) == ((-1, -1, -1), (66, 66, 66))
    assert geometry.environment_window((0, 0, 0, 63, 63, 63), (0, 0, 0), 0.5) == ((-1, -1, -1), (128, 128, 128))


def test_custom_catalog_matches_the_reference_build(oracle_ref):
    # The reference's make_orientation_catalog in catalog mode
    # (orientations.cpp:104-172): unit length, the w > 0 sign rule, and
    # first-seen de-duplication, on seeded quaternions with scaled copies,
    # sign flips and w = 0 entries mixed in.
    geometry = package("geometry")
    rng = np.random.default_rng(12)
    q = rng.standard_normal((40, 4))
    q[5] = -q[3]
    q[9] = 3.5 * q[1]
    q[12] = [0.0, 0.6, -0.8, 0.0]
    q[13] = [0.0, -0.6, 0.8, 0.0]
    q[20] = [1e-3, 0.0, 0.0, 0.0]
    got = geometry.custom_catalog(q)
    want = oracle_ref.catalog(4, q)
    assert got.shape == want.shape
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
