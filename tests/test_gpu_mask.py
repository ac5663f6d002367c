"""Device-thresholded binary correlation (spk_correlate_binary_mask) against
the mask oracle, and against the counts of spk_correlate_binary on the same
inputs.  Masks are bit-exact: they come from integer counts."""

import numpy as np
import pytest

from conftest import package
from oracle import masks

pytestmark = pytest.mark.gpu


def _case(rng, max_env=20, max_ker=8):
    es = rng.integers(1, max_env, size=3)
    ks = rng.integers(1, max_ker, size=3)
    ef = rng.integers(-30, 30, size=3)
    kf = rng.integers(-30, 30, size=3)
    env = (rng.random(int(np.prod(es))) < rng.random()).astype(np.uint8)
    ker = (rng.random(int(np.prod(ks))) < 0.5).astype(np.uint8)
    ker[0] = 1
    return es, ks, ef, kf, env, ker


def _boxes(es, ks, ef, kf, tf, shape):
    legal = ([int(ef[a]) - int(kf[a]) for a in range(3)], [max(int(es[a]) - int(ks[a]) + 1, 0) for a in range(3)])
    wide = ([int(tf[a]) - 3 for a in range(3)], [int(shape[a]) + 5 for a in range(3)])
    full = ([int(v) for v in tf], [int(v) for v in shape])
    return legal, wide, full


@pytest.mark.parametrize("precision", [0, 1])
def test_masks_match_oracle(gpu_ctx, oracle_c, precision):
    compute = package("compute")
    rng = np.random.default_rng(300 + precision)
    for _ in range(20):
        es, ks, ef, kf, env, ker = _case(rng)
        spec = compute.CorrelationSpec(es, ks, ef, kf)
        tf, shape, values = oracle_c.correlate(False, es, ks, ef, kf, env, ker)
        for first, bshape in _boxes(es, ks, ef, kf, tf, shape):
            for select in (compute.MASK_ZERO, compute.MASK_NONZERO):
                got = compute.correlate_binary_mask(spec, env, ker, first, bshape, select, precision=precision,
                                                    context=gpu_ctx)
                assert isinstance(got, compute.MaskResult), got
                assert list(got.translation_first) == list(tf) and list(got.shape) == list(shape)
                want = masks.translation_mask(tf, shape, values, first, bshape, select == compute.MASK_ZERO)
                assert np.array_equal(got.mask, want), (es, ks, first, bshape, select)


def _balls(rng, side, count, radius):
    zz, yy, xx = np.mgrid[0:side, 0:side, 0:side]
    field = np.zeros((side, side, side), bool)
    for _ in range(count):
        c = rng.uniform(0, side, 3)
        r = rng.uniform(radius / 2, radius)
        field |= (xx - c[0]) ** 2 + (yy - c[1]) ** 2 + (zz - c[2]) ** 2 < r * r
    return field.astype(np.uint8).reshape(-1)


def test_gap_fill_shapes_match_the_counts_path(gpu_ctx):
    # A box-scale environment with placed copies and a ball kernel: the free
    # mask over the legal box, and the blocked mask over the full range.
    compute = package("compute")
    rng = np.random.default_rng(5)
    es, ks = np.array([80, 80, 80]), np.array([24, 24, 24])
    ef, kf = np.array([-1, -1, -1]), np.array([-12, -12, -12])
    env = _balls(rng, 80, 12, 14)
    ker = _balls(np.random.default_rng(6), 24, 1, 12)
    spec = compute.CorrelationSpec(es, ks, ef, kf)
    full = compute.correlate_binary(spec, env, ker, precision=compute.FP64, context=gpu_ctx)
    assert isinstance(full, compute.CorrelationResult), full
    for first, bshape, select in (([int(ef[a] - kf[a]) for a in range(3)], [57, 57, 57], compute.MASK_ZERO),
                                  (list(full.translation_first), list(full.shape), compute.MASK_NONZERO)):
        got = compute.correlate_binary_mask(spec, env, ker, first, bshape, select, precision=compute.FP64,
                                            context=gpu_ctx)
        assert isinstance(got, compute.MaskResult), got
        want = masks.translation_mask(full.translation_first, full.shape, full.values, first, bshape,
                                      select == compute.MASK_ZERO)
        assert np.array_equal(got.mask, want)
        assert 0 < int(got.mask.sum()) < got.mask.size
        # Same kernels on the same inputs: the same checks, value for value.
        assert got.numeric == full.numeric


def test_refusals_match_the_counts_path(gpu_ctx):
    # FP16 spectra are refused by the mass or probe checks at most sizes;
    # whatever spk_correlate_binary answers, the mask variant answers too.
    compute = package("compute")
    rng = np.random.default_rng(9)
    for _ in range(6):
        es, ks, ef, kf, env, ker = _case(rng, max_env=40, max_ker=12)
        spec = compute.CorrelationSpec(es, ks, ef, kf)
        counts = compute.correlate_binary(spec, env, ker, precision=compute.FP16, context=gpu_ctx)
        tf = counts.translation_first if isinstance(counts, compute.CorrelationResult) else \
            [int(ef[a]) - int(kf[a]) - (int(ks[a]) - 1) for a in range(3)]
        shape = [int(es[a]) + int(ks[a]) - 1 for a in range(3)]
        got = compute.correlate_binary_mask(spec, env, ker, tf, shape, compute.MASK_NONZERO,
                                            precision=compute.FP16, context=gpu_ctx)
        if isinstance(counts, compute.CorrelationFailure):
            assert isinstance(got, compute.CorrelationFailure) and got.code == counts.code
        else:
            assert isinstance(got, compute.MaskResult)
            assert np.array_equal(got.mask, masks.translation_mask(tf, shape, counts.values, tf, shape, False))


def test_invalid_requests_are_rejected(gpu_ctx):
    compute, lib_mod = package("compute"), package("_lib")
    rng = np.random.default_rng(10)
    es, ks, ef, kf, env, ker = _case(rng)
    spec = compute.CorrelationSpec(es, ks, ef, kf)
    with pytest.raises(lib_mod.SpkError):
        compute.correlate_binary_mask(spec, env, ker, (0, 0, 0), (4, 4, 4), context=gpu_ctx, capacity=63)
    with pytest.raises(lib_mod.SpkError):
        compute.correlate_binary_mask(spec, env, ker, (0, 0, 0), (4, 4, 4), select=2, context=gpu_ctx)
