"""A session's occupancy and proximity after each placement against the
reference build's own fields for the same layout (its BlockedField::add and
build_proximity, observed on a page of its spectral pipeline).

A session places copies through the device placement path: for a pose
whose rotation is not cardinal, the vertex intervals and their bounds are
computed on the device; for every pose, the face ranges and their offsets
are.  The fields must be bit-exact all the same: a blob at seeded general
rotations (device intervals), and a cuboid at the 24 cube rotations (host
intervals, device face ranges), placed at the reference's own chosen
translations.
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


@pytest.mark.parametrize("item", ["blob", "cuboid"])
def test_session_fields_match_reference_after_each_placement(gpu_ctx, oracle_ref, item):
    assets, geometry, session_mod = package("assets"), package("geometry"), package("session")
    if item == "blob":
        stl = syn.blob_stl(13, level=4, radius_range=(3.0, 5.5))
        raw = _rotations(np.random.default_rng(13), 6)
        box = (40.0, 34.0, 30.0)
        catalog = oracle_ref.catalog(4, raw)
    else:
        stl = syn.cuboid_stl((7.0, 5.5, 4.25))
        box = (36.0, 30.0, 26.0)
        catalog = oracle_ref.catalog(1)
    ref = oracle_ref.session(oracle_ref.asset(stl), box, 0.0, 0.0, (0.0, 0.0, 0.0), 1.0, catalog)
    s = session_mod.Session(assets.accept_stl(stl), box, (0.0, 0.0, 0.0), 1.0, catalog, context=gpu_ctx)
    assert np.array_equal(s.catalog, catalog)
    placed = 0
    for step in range(8):
        page = ref.page(step % len(catalog))
        if not page or not ref.place(page[0].orientation, list(page[0].t)):
            continue
        s.place(page[0].orientation, tuple(page[0].t))
        placed += 1
        ref.page(0, keep_values=True)
        occ_ref, meta = ref.observed(0)
        prox_ref, _ = ref.observed(1)
        occ = s.field("occupancy")
        first, shape = s.last_window
        assert list(first) == list(meta[0]) and list(shape) == list(meta[1])
        assert np.array_equal(occ, occ_ref), (item, step)
        prox = s.field("proximity")
        assert np.array_equal(prox.view(np.uint64), prox_ref.view(np.uint64)), (item, step)
    assert placed >= 4
    s.close()
