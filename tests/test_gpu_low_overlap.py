"""Low-overlap pages (CandidatePageMode::low_overlap, spectral_pipeline.cpp:
1758-1824) against the reference build's own pages.

The reference ranks every legal translation, colliding ones included, by
(rounded binary overlap, score, orientation, z, y, x) and returns 32 after
the cursor, with no direct recount.  The GPU page must hold the same
translations with the same overlap counts, and scores equal up to the
reference's FFT rounding; among candidates with the same count whose scores
are that close, the order is the reference's FFT noise and may differ.
Three pages are walked per orientation by each side's own cursor, on
layouts of a few copies in boxes tight enough that the pages run from zero
counts into collisions (seed 3) or hold collisions only (seed 4).
"""

import importlib

import numpy as np
import pytest

from conftest import package

pytestmark = pytest.mark.gpu
syn = importlib.import_module("cpp-max-packer_b200.synthetic")
TOL = 1e-9


def _catalog(rng, n):
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1)[:, None]
    q[q[:, 3] < 0] *= -1
    return q


def _groups(entries):
    """Runs of equal (count, score within TOL) as sets of translations."""
    out = []
    for t, score, count in entries:
        if out and out[-1][0] == count and abs(out[-1][1] - score) < TOL:
            out[-1][2].add(t)
        else:
            out.append([count, score, {t}])
    return out


@pytest.mark.parametrize("seed,box", [(3, (18.0, 15.0, 13.0)), (4, (22.0, 18.0, 15.0))])
def test_low_overlap_pages_match_reference(gpu_ctx, oracle_ref, seed, box):
    assets, session_mod = package("assets"), package("session")
    rng = np.random.default_rng(seed)
    stl = syn.blob_stl(seed, level=2, radius_range=(3.0, 4.5))
    catalog = oracle_ref.catalog(4, _catalog(rng, 4))
    ref = oracle_ref.session(oracle_ref.asset(stl), box, 0.0, 0.0, (0.0, 0.0, 0.0), 1.0, catalog)
    s = session_mod.Session(assets.accept_stl(stl), box, (0.0, 0.0, 0.0), 1.0, catalog, context=gpu_ctx)
    assert np.array_equal(s.catalog, catalog)
    for step in range(4):
        page = ref.page(step % len(catalog))
        if page and ref.place(page[0].orientation, list(page[0].t)):
            s.place(page[0].orientation, tuple(page[0].t))
    collisions = 0
    for o in range(len(catalog)):
        ref_cursor, gpu_cursor = None, None
        ref_all, gpu_all = [], []
        for _ in range(3):
            ref_page = ref.page(o, cursor=ref_cursor, low_overlap=True)
            gpu_page = s.pages([o], cursors=[gpu_cursor], low_overlap=True)[0]
            assert len(gpu_page) == len(ref_page)
            if not ref_page:
                break
            for r, g in zip(ref_page, gpu_page):
                assert g.orientation_index == r.orientation == o
                assert g.binary_overlap == r.binary_overlap == round(r.binary_overlap)
                assert abs(g.score - r.score) < TOL
                assert not g.direct_zero_overlap and not r.direct_zero
            ref_all += [(tuple(r.t), r.score, r.binary_overlap) for r in ref_page]
            gpu_all += [(tuple(g.translation), g.score, g.binary_overlap) for g in gpu_page]
            ref_cursor, gpu_cursor = ref_page[-1], gpu_page[-1]
        counts = [c for _, _, c in gpu_all]
        assert counts == sorted(counts)
        collisions += sum(c > 0 for c in counts)
        ref_groups, gpu_groups = _groups(ref_all), _groups(gpu_all)
        assert len(ref_groups) == len(gpu_groups)
        # every group but the last (which the page boundary may cut) has the same members
        for a, b in zip(ref_groups[:-1], gpu_groups[:-1]):
            assert a[0] == b[0] and a[2] == b[2]
    assert collisions > 0
    s.close()
