"""The incremental EDT of a placement session against a full rebuild.

After a copy is placed on an up-to-date layout, the session updates the
squared distances in place: only the box of tiles whose largest squared
distance the new copy could lower is recomputed, as the minimum of the old
value and the squared distance to the copy's cells.  After every placement of
a greedy fill its proximity field must equal, bit for bit, the full
spk_build_proximity (the reference's build_proximity,
field_proximity.hpp:32-132) of the same occupancy.  Removing a copy rebuilds
the field from scratch, which the same comparison covers.
"""

import numpy as np
import pytest

from conftest import package

pytestmark = pytest.mark.gpu


def _fill_and_compare(gpu_ctx, wl, steps):
    session_mod, compute = package("session"), package("compute")
    s = session_mod.Session(wl.obj, wl.container, wl.origin, wl.pitch, wl.catalog, wl.pair_clearance,
                            wl.wall_clearance, context=gpu_ctx)
    shape = s.environment_shape
    checked = 0
    for i in range(steps):
        if not s.greedy(1):
            break
        prox = s.field("proximity")
        occ = s.field("occupancy")
        full = compute.build_proximity(shape, occ, context=gpu_ctx)
        assert np.array_equal(prox, full), f"step {i}: incremental proximity differs from the full rebuild"
        checked += 1
    # A removal, then a placement on the rebuilt field.
    s.remove_last()
    assert np.array_equal(s.field("proximity"),
                          compute.build_proximity(shape, s.field("occupancy"), context=gpu_ctx))
    s.greedy(1)
    assert np.array_equal(s.field("proximity"),
                          compute.build_proximity(shape, s.field("occupancy"), context=gpu_ctx))
    s.close()
    return checked


def test_incremental_edt_blob128(gpu_ctx):
    # The 63 mm box holds about 30 copies of this blob in 8 orientations.
    wl = package("workloads").box63_blob_hopf96()
    wl.catalog = wl.catalog[:8]
    assert _fill_and_compare(gpu_ctx, wl, 60) >= 25


def test_incremental_edt_cuboid66(gpu_ctx):
    wl = package("workloads").box64_cuboid_cube24()
    assert _fill_and_compare(gpu_ctx, wl, 80) >= 40


def test_incremental_edt_rounded256(gpu_ctx):
    wl = package("workloads").rounded256_blob_hopf512(orientations=8)
    assert _fill_and_compare(gpu_ctx, wl, 60) == 60
