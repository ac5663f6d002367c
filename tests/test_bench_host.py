"""bench.py's whole-step model figures, checked by hand on the host."""

import math

import pytest


def test_step_model_at_256_cubed_with_512_orientations():
    import bench

    m = bench.step_model((256, 256, 256), (256, 256, 256), 512, 100.0, 6500.0)
    ph = 129 * 256 * 256
    want = 24 * ph * 512 + 64 * ph + 26 * 256 ** 3
    assert m["model_bytes_per_step"] == want  # about 104.9 GB
    assert m["achieved"] == pytest.approx(want / 0.1 / 1e9, abs=0.05)
    assert m["frac"] == pytest.approx(m["achieved"] / 6500.0, abs=1e-4)
    assert m["floor_ms_per_step"] == pytest.approx(want / 6.5e12 * 1e3, abs=1e-3)
    p = 256 ** 3
    assert m["fft_flops_per_step"] == pytest.approx(2.5 * p * math.log2(p) * 1026)


def test_step_model_with_no_time_or_peak_reports_no_rate():
    import bench

    m = bench.step_model((2, 2, 2), (2, 2, 2), 1, 0.0, 0.0)
    assert m["achieved"] == 0.0 and m["frac"] is None and m["floor_ms_per_step"] is None
