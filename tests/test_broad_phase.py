"""Validator broad phase: posed bounds and the outward-AABB pair test
(engine/pack_geometry/src/validation.cpp:404-418, validation_kernel.cpp:
1000-1088 and 1245-1261).

CPU: the host posed bounds (spk_posed_bounds) with the oracle's pair test
(oracle_broad_phase) against the reference build's own
bounds_pair_certificate, on pose pairs placed so that their bounds touch,
nearly touch or nearly overlap within a few ulps, for a blob (general
rotations) and a cuboid (cardinal rotations), with and without clearance.

GPU: spk_broad_phase against oracle_broad_phase on layouts of up to 3,000
copies (bounds with exact ties), with proven copies and with an output
capacity below the unresolved count.
"""

import importlib

import numpy as np
import pytest

from conftest import package

syn = importlib.import_module("cpp-max-packer_b200.synthetic")


def _quaternions(rng, n, cardinal):
    if cardinal:
        geometry = package("geometry")
        cube = geometry.cube_catalog()
        return cube[rng.integers(0, len(cube), size=n)]
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1)[:, None]
    q[q[:, 3] < 0] *= -1
    return q


@pytest.mark.parametrize("item,cardinal,clearance", [("blob", False, 0.0), ("blob", False, 0.35),
                                                     ("cuboid", True, 0.0), ("cuboid", True, 0.2),
                                                     ("cuboid", False, 0.1)])
def test_pair_test_matches_reference_certificate(oracle_c, oracle_ref, item, cardinal, clearance):
    assets, geometry = package("assets"), package("geometry")
    stl = syn.blob_stl(5, level=2, radius_range=(3.0, 4.5)) if item == "blob" else syn.cuboid_stl((7.0, 4.5, 3.25))
    mesh = assets.accept_stl(stl)
    ref_asset = oracle_ref.asset(stl)
    rng = np.random.default_rng(len(item) * 10 + int(cardinal) + int(clearance * 100))
    checked = certified = 0
    for trial in range(40):
        q = _quaternions(rng, 2, cardinal)
        t0 = rng.uniform(-20, 20, size=3)
        lo0, hi0, f0 = geometry.posed_bounds(mesh, [t0], [q[0]])
        axis = int(rng.integers(0, 3))
        # Second copy's bounds at the origin, then moved along `axis` so that
        # its min lands on first max + clearance, give or take a few ulps.
        lo1z, _, _ = geometry.posed_bounds(mesh, [[0.0, 0.0, 0.0]], [q[1]])
        base = hi0[0, axis] + clearance - lo1z[0, axis]
        for step in (-3, -1, 0, 1, 2, 4):
            t1 = t0 + rng.uniform(-1, 1, size=3) * 0.5
            t1[axis] = np.nextafter(base, np.inf) if step == 0 else base + step * np.spacing(base) * 3
            lo, hi, fin = geometry.posed_bounds(mesh, [t0, t1], [q[0], q[1]])
            pairs, count = oracle_c.broad_phase(lo, hi, fin, None, clearance)
            ref = ref_asset.bounds_pair(t1, q[1], t0, q[0], clearance)
            assert ref in (0, 1, 2), ref
            # pair (first=1, second=0) is unresolved exactly when the reference
            # does not certify it by the outward AABBs
            assert (count == 1) == (ref != 1), (trial, step, ref, lo, hi)
            checked += 1
            certified += ref == 1
    assert 0 < certified < checked


def test_oracle_visiting_order_and_proven(oracle_c):
    # Three overlapping unit boxes and one far away: pairs (1,0), (2,0), (2,1)
    # unresolved in that order; proven copies 0 and 1 drop (1,0).
    lo = np.array([[0, 0, 0], [0.5, 0, 0], [0.2, 0.2, 0.2], [10, 10, 10]], np.float64)
    hi = lo + 1.0
    fin = np.ones(4, np.uint8)
    pairs, count = oracle_c.broad_phase(lo, hi, fin, None, 0.0)
    assert count == 3 and pairs.tolist() == [[1, 0], [2, 0], [2, 1]]
    pairs, count = oracle_c.broad_phase(lo, hi, fin, np.array([1, 1, 0, 0], np.uint8), 0.0)
    assert pairs.tolist() == [[2, 0], [2, 1]]
    # a copy without finite bounds certifies nothing
    fin[3] = 0
    pairs, count = oracle_c.broad_phase(lo, hi, fin, None, 0.0)
    assert count == 6 and pairs[-3:].tolist() == [[3, 0], [3, 1], [3, 2]]


def _layout(rng, n):
    """Bounds on a coarse lattice so that many faces touch exactly."""
    lo = rng.integers(0, 40, size=(n, 3)).astype(np.float64) * 0.5
    hi = lo + rng.integers(1, 5, size=(n, 3)).astype(np.float64) * 0.5
    fin = (rng.random(n) > 0.01).astype(np.uint8)
    return lo, hi, fin


@pytest.mark.gpu
@pytest.mark.parametrize("n,clearance,with_proven", [(2, 0.0, False), (300, 0.0, False), (1000, 0.25, True),
                                                     (3000, 0.5, True)])
def test_device_broad_phase_matches_oracle(gpu_ctx, oracle_c, n, clearance, with_proven):
    geometry = package("geometry")
    rng = np.random.default_rng(n)
    lo, hi, fin = _layout(rng, n)
    proven = (np.arange(n) < n * 3 // 4).astype(np.uint8) if with_proven else None
    want, count = oracle_c.broad_phase(lo, hi, fin, proven, clearance)
    got = geometry.broad_phase(lo, hi, fin, clearance, proven=proven, context=gpu_ctx)
    assert got.shape == want.shape and np.array_equal(got, want), (got[:5], want[:5])
    assert 0 < count < n * (n - 1) // 2 or n == 2


@pytest.mark.gpu
def test_device_broad_phase_capacity(gpu_ctx, oracle_c):
    geometry, lib_mod = package("geometry"), package("_lib")
    rng = np.random.default_rng(7)
    lo, hi, fin = _layout(rng, 400)
    want, count = oracle_c.broad_phase(lo, hi, fin, None, 0.0)
    with pytest.raises(lib_mod.SpkError) as err:
        geometry.broad_phase(lo, hi, fin, 0.0, context=gpu_ctx, capacity=count - 1)
    assert err.value.status == 25
    got = geometry.broad_phase(lo, hi, fin, 0.0, context=gpu_ctx, capacity=count)
    assert np.array_equal(got, want)


@pytest.mark.gpu
def test_device_broad_phase_on_posed_layout(gpu_ctx, oracle_c, oracle_ref):
    # Posed bounds of a packed layout: the GPU session's own placements of
    # blobs, whose bounds overlap where the copies nest.
    assets, geometry, session_mod, workloads = (package("assets"), package("geometry"), package("session"),
                                                package("workloads"))
    wl = workloads.rounded256_blob_hopf512(orientations=16)
    s = session_mod.Session(wl.obj, wl.container, wl.origin, wl.pitch, wl.catalog, context=gpu_ctx)
    placed = s.greedy(24)
    s.close()
    t = np.array([[wl.origin[a] + wl.pitch * p.translation[a] for a in range(3)] for p in placed])
    q = np.array([wl.catalog[p.orientation_index] for p in placed])
    lo, hi, fin = geometry.posed_bounds(wl.obj, t, q)
    want, count = oracle_c.broad_phase(lo, hi, fin, None, 0.0)
    got = geometry.broad_phase(lo, hi, fin, 0.0, context=gpu_ctx)
    assert np.array_equal(got, want) and count > 0
    # and the reference's own certificate for every pair of the layout
    ref_asset = oracle_ref.asset(wl.object_stl)
    unresolved = {tuple(p) for p in got.tolist()}
    for first in range(len(t)):
        for second in range(first):
            ref = ref_asset.bounds_pair(t[first], q[first], t[second], q[second], 0.0)
            assert ((first, second) in unresolved) == (ref != 1)
