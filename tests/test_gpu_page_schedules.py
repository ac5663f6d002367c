"""The 256^3 page passes under each launch schedule give the same pages.

The default runs passes A, B1 and B2 as one launch each per batch of 16
orientations. SPK_PAGE_SCHEDULE=staged pipelines them (pass A of batch k with
B1 of k - 1 and B2 of k - 2 in one launch, three intermediates in rotation),
and SPK_PASS_B=fused runs B1 and B2 as one cluster kernel per orientation.
The schedule is read when a session's pipeline is built. The check pages 48
orientations of the bench workload (three batches) and 40 (a last batch of
8) after a few placements, under each schedule, and compares every candidate
and the residual bit for bit.
"""

import pytest

from conftest import package

pytestmark = pytest.mark.gpu


def _pages(monkeypatch, gpu_ctx, env, orientations):
    for name in ("SPK_PAGE_SCHEDULE", "SPK_PASS_B"):
        monkeypatch.delenv(name, raising=False)
    for name, value in env.items():
        monkeypatch.setenv(name, value)
    session_mod, workloads = package("session"), package("workloads")
    wl = workloads.rounded256_blob_hopf512(orientations=orientations)
    s = session_mod.Session(wl.obj, wl.container, wl.origin, wl.pitch, wl.catalog, context=gpu_ctx)
    placed = s.greedy(3)
    reports = []
    pages = s.pages(range(orientations), reports=reports)
    s.close()
    return [(p.orientation_index, p.translation) for p in placed], pages, reports


@pytest.mark.timeout(900)
@pytest.mark.parametrize("orientations", [48, 40])
def test_page_schedules_agree(monkeypatch, gpu_ctx, orientations):
    placed, pages, reports = _pages(monkeypatch, gpu_ctx, {}, orientations)
    assert len(placed) == 3 and sum(len(p) for p in pages) > 0
    for env in ({"SPK_PAGE_SCHEDULE": "staged"}, {"SPK_PASS_B": "fused"}):
        other_placed, other_pages, other_reports = _pages(monkeypatch, gpu_ctx, env, orientations)
        assert other_placed == placed, env
        assert other_pages == pages, env
        for a, b in zip(reports, other_reports):
            assert a["max_integer_residual"] == b["max_integer_residual"], env
