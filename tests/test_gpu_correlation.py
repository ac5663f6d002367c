"""GPU full-range correlation and proximity field against the oracle."""

import numpy as np
import pytest

from conftest import package

pytestmark = pytest.mark.gpu


def _case(rng, proximity, max_env=24, max_ker=9):
    es = rng.integers(1, max_env, size=3)
    ks = rng.integers(1, max_ker, size=3)
    ef = rng.integers(-40, 40, size=3)
    kf = rng.integers(-40, 40, size=3)
    n = int(np.prod(es))
    env = rng.random(n) if proximity else (rng.random(n) < rng.random()).astype(np.uint8)
    ker = (rng.random(int(np.prod(ks))) < 0.5).astype(np.uint8)
    ker[0] = 1
    return es, ks, ef, kf, env, ker


@pytest.mark.parametrize("precision", [0, 1])
def test_binary_matches_oracle_exactly(gpu_ctx, oracle_c, precision):
    compute = package("compute")
    rng = np.random.default_rng(100 + precision)
    for _ in range(30):
        es, ks, ef, kf, env, ker = _case(rng, False)
        spec = compute.CorrelationSpec(es, ks, ef, kf)
        got = compute.correlate_binary(spec, env, ker, precision=precision, context=gpu_ctx)
        tf, shape, want = oracle_c.correlate(False, es, ks, ef, kf, env, ker)
        assert isinstance(got, compute.CorrelationResult), got
        assert list(got.translation_first) == list(tf) and list(got.shape) == list(shape)
        assert np.array_equal(got.values, want)
        assert got.numeric.max_integer_residual < 0.25


def test_proximity_fp64_within_reference_tolerance(gpu_ctx, oracle_c):
    compute = package("compute")
    rng = np.random.default_rng(7)
    for _ in range(30):
        es, ks, ef, kf, env, ker = _case(rng, True)
        spec = compute.CorrelationSpec(es, ks, ef, kf)
        got = compute.correlate_proximity(spec, env, ker, precision=compute.FP64, context=gpu_ctx)
        tf, shape, want = oracle_c.correlate(True, es, ks, ef, kf, env, ker)
        assert isinstance(got, compute.CorrelationResult), got
        # The reference's own tolerance (correlation.cpp:493,573).
        assert np.all(np.abs(got.values - want) <= 1e-10 * np.maximum(1.0, np.abs(want)))


def test_proximity_fp32_within_stated_bound(gpu_ctx, oracle_c):
    compute = package("compute")
    rng = np.random.default_rng(8)
    for _ in range(10):
        es, ks, ef, kf, env, ker = _case(rng, True)
        got = compute.correlate_proximity(compute.CorrelationSpec(es, ks, ef, kf), env, ker,
                                          precision=compute.FP32, context=gpu_ctx)
        _, _, want = oracle_c.correlate(True, es, ks, ef, kf, env, ker)
        assert isinstance(got, compute.CorrelationResult), got
        # FP32 bound stated by the path: 2^-13 of the output scale.
        assert np.abs(got.values - want).max() <= max(1.0, want.max()) / 8192


def test_golden_cases_through_gpu(gpu_ctx):
    compute = package("compute")
    # engine/pack_compute/tests/correlation_tests.cpp:292-308
    r = compute.correlate_binary(compute.CorrelationSpec((3, 2, 1), (2, 2, 1), (4, -3, 0), (-1, 1, 0)),
                                 [1, 0, 1, 0, 1, 1], [1, 0, 1, 1], context=gpu_ctx)
    assert r.translation_first == (4, -5, 0) and r.shape == (4, 3, 1)
    # correlation_tests.cpp:310-327
    r = compute.correlate_proximity(compute.CorrelationSpec((2, 1, 1), (2, 1, 1), (9, 0, 0), (3, 0, 0)),
                                    [0.5, 1.0], [1, 1], context=gpu_ctx)
    assert r.translation_first == (5, 0, 0)
    assert np.allclose(r.values, [0.5, 1.5, 1.0], atol=1e-12)
    # correlation_tests.cpp:350-364: padded-cell admission before allocation
    limits = compute.CorrelationLimits(max_padded_cells=100)
    r = compute.correlate_binary(compute.CorrelationSpec((3, 3, 3), (3, 3, 3)), np.ones(27), np.ones(27),
                                 limits=limits, context=gpu_ctx)
    assert isinstance(r, compute.CorrelationFailure) and r.code == "CORRELATION_PADDED_CELL_LIMIT"
    # invalid inputs fail as values
    r = compute.correlate_binary(compute.CorrelationSpec((2, 1, 1), (1, 1, 1)), [2, 0], [1], context=gpu_ctx)
    assert r.code == "CORRELATION_INVALID_ENVIRONMENT"
    r = compute.correlate_binary(compute.CorrelationSpec((2, 1, 1), (1, 1, 1)), [1, 0], [3], context=gpu_ctx)
    assert r.code == "CORRELATION_INVALID_KERNEL"


def test_stop_and_deadline_return_codes(gpu_ctx):
    compute = package("compute")
    control = compute.OperationControl()
    control.request_stop()
    r = compute.correlate_binary(compute.CorrelationSpec((4, 4, 4), (2, 2, 2)), np.ones(64), np.ones(8),
                                 control=control, context=gpu_ctx)
    assert r.code == "OPERATION_CANCELLED"
    r = compute.correlate_binary(compute.CorrelationSpec((4, 4, 4), (2, 2, 2)), np.ones(64), np.ones(8),
                                 control=compute.OperationControl(deadline_ns=1), context=gpu_ctx)
    assert r.code == "DEADLINE_EXCEEDED"


@pytest.mark.parametrize("axis_len", [13, 127])
def test_general_lengths_every_axis(gpu_ctx, oracle_c, axis_len):
    # correlation_tests.cpp:466-481 qualify lengths 13 (8+6-1) and 127 (64+64-1)
    compute = package("compute")
    e, k = (8, 6) if axis_len == 13 else (64, 64)
    rng = np.random.default_rng(axis_len)
    for axis in range(3):
        es = [3, 3, 3]
        ks = [2, 2, 2]
        es[axis], ks[axis] = e, k
        env = (rng.random(int(np.prod(es))) < 0.5).astype(np.uint8)
        ker = (rng.random(int(np.prod(ks))) < 0.5).astype(np.uint8)
        ker[0] = 1
        got = compute.correlate_binary(compute.CorrelationSpec(es, ks), env, ker, context=gpu_ctx)
        _, _, want = oracle_c.correlate(False, es, ks, (0, 0, 0), (0, 0, 0), env, ker)
        assert np.array_equal(got.values, want)


def test_proximity_field_bit_exact(gpu_ctx, oracle_c):
    compute = package("compute")
    rng = np.random.default_rng(21)
    for shape in [(1, 1, 1), (7, 5, 3), (33, 17, 9), (66, 66, 66), (128, 96, 64)]:
        for density in (0.0, 0.001, 0.2):
            occ = (rng.random(int(np.prod(shape))) < density).astype(np.uint8)
            got = compute.build_proximity(shape, occ, context=gpu_ctx)
            want, _ = oracle_c.build_proximity(shape, occ)
            assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), shape


def test_proximity_long_lines_bit_exact(gpu_ctx, oracle_c):
    # Lines of 256 and 512 cells (the shared-memory envelope's range) and one
    # beyond it (the global-memory pass), with sparse sites, dense sites and
    # runs of occupied cells.
    compute = package("compute")
    rng = np.random.default_rng(22)
    for shape in [(256, 200, 40), (40, 256, 33), (17, 23, 512), (600, 9, 7), (1100, 5, 3), (1, 300, 2)]:
        n = int(np.prod(shape))
        for density in (0.0005, 0.05, 0.7):
            occ = (rng.random(n) < density).astype(np.uint8)
            got = compute.build_proximity(shape, occ, context=gpu_ctx)
            want, _ = oracle_c.build_proximity(shape, occ)
            assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), (shape, density)


def _blob(shape, rng):
    zz, yy, xx = np.mgrid[0:shape[2], 0:shape[1], 0:shape[0]]
    c = (np.array(shape) - 1) / 2
    d = ((xx - c[0]) / (shape[0] / 2)) ** 2 + ((yy - c[1]) / (shape[1] / 2)) ** 2 + ((zz - c[2]) / (shape[2] / 2)) ** 2
    return (d + rng.normal(0, 0.1, d.shape) < 1).astype(np.uint8).reshape(-1)


def test_fp16_spectra_fail_closed_or_exact(gpu_ctx, oracle_c):
    # FP16 spectra round the DC term by ~2^-11 of the overlap mass, so the
    # reference's mass check (sum of unrounded counts within 0.25 of the exact
    # mass) refuses them beyond tiny fields; whatever is returned is exact.
    compute = package("compute")
    rng = np.random.default_rng(31)
    cases = [((6, 6, 5), (3, 1, 1), 0.2, True), ((20, 18, 16), (4, 5, 3), 0.3, False),
             ((33, 9, 12), (6, 3, 5), 0.3, False)]
    for es, ks, density, must_pass in cases:
        env = (rng.random(int(np.prod(es))) < density).astype(np.uint8)
        ker = _blob(ks, rng) if min(ks) > 1 else np.ones(int(np.prod(ks)), np.uint8)
        got = compute.correlate_binary(compute.CorrelationSpec(es, ks), env, ker, precision=compute.FP16,
                                       context=gpu_ctx)
        _, _, want = oracle_c.correlate(False, es, ks, (0, 0, 0), (0, 0, 0), env, ker)
        if isinstance(got, compute.CorrelationResult):
            assert np.array_equal(got.values, want)
        else:
            assert not must_pass and got.code == "CORRELATION_NUMERIC", got


def test_fp16_spectra_proximity_within_stated_bound(gpu_ctx, oracle_c):
    # Real-valued proximity correlations with FP16 spectra: values within
    # 2^-8 of the output scale (the largest possible output) of the exact result.
    compute = package("compute")
    rng = np.random.default_rng(33)
    for es, ks in [((24, 20, 18), (5, 4, 3)), ((40, 40, 40), (7, 7, 7))]:
        env = rng.random(int(np.prod(es)))
        ker = _blob(ks, rng)
        got = compute.correlate_proximity(compute.CorrelationSpec(es, ks), env, ker, precision=compute.FP16,
                                          context=gpu_ctx)
        _, _, want = oracle_c.correlate(True, es, ks, (0, 0, 0), (0, 0, 0), env, ker)
        assert isinstance(got, compute.CorrelationResult), got
        # The stated FP16 scale: 2^-8 of the largest possible output, min(environment mass, kernel cells).
        assert np.abs(got.values - want).max() <= max(1.0, min(env.sum(), float(ker.sum()))) / 256


def test_fp16_spectra_refused_at_the_medium_scale(gpu_ctx):
    # A 128^3 half-occupied environment against a 21^3 blob: FP64 (pinned to
    # the oracle on smaller fields) passes the reference's checks; FP16 spectra
    # exceed the integer bound and are refused.
    compute = package("compute")
    rng = np.random.default_rng(32)
    es, ks = (128, 128, 128), (21, 21, 21)
    env = (rng.random(int(np.prod(es))) < 0.5).astype(np.uint8)
    ker = _blob(ks, rng)
    spec = compute.CorrelationSpec(es, ks)
    lim = compute.CorrelationLimits(max_working_bytes=4 << 30)  # the FP64 grid alone is 537 MB
    want = compute.correlate_binary(spec, env, ker, limits=lim, precision=compute.FP64, context=gpu_ctx)
    got32 = compute.correlate_binary(spec, env, ker, limits=lim, precision=compute.FP32, context=gpu_ctx)
    got16 = compute.correlate_binary(spec, env, ker, limits=lim, precision=compute.FP16, context=gpu_ctx)
    assert isinstance(want, compute.CorrelationResult)
    # FP32 passes the reference's checks or is refused by them (at this mass the
    # 0.25 mass check is beyond FP32 accumulation); it is never wrong.
    if isinstance(got32, compute.CorrelationResult):
        assert np.array_equal(got32.values, want.values)
    else:
        assert got32.code == "CORRELATION_NUMERIC", got32
    assert isinstance(got16, compute.CorrelationFailure) and got16.code == "CORRELATION_NUMERIC", got16
