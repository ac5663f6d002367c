"""Transform lengths other than powers of two.

The shared-memory FFT takes every 2^a 3^b 5^c length up to 512 (radix 4, 2,
3 and 5 stages), and the page pipeline's lengths are chosen per window by the
autotuner among the supported lengths from the window's extent up to the next
power of two.  These tests check:

- the full-range drop-in correlation on padded extents that are not powers of
  two (its transform length is the smallest supported one), against the
  exact integer oracle;
- that pages and greedy sequences on windows of 130, 150 and 192 cells per
  axis are identical with the tuned lengths and with power-of-two lengths
  (SPK_FFT_LENGTHS=pow2), since the certified pages are exact either way;
- one odd window's page against the oracle's page restatement.
"""

import os

import numpy as np
import pytest

from conftest import package

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("es,ks", [((20, 21, 13), (6, 5, 3)), ((40, 27, 31), (9, 10, 5)), ((61, 7, 50), (15, 3, 11))])
def test_drop_in_on_smooth_lengths(gpu_ctx, oracle_c, es, ks):
    compute = package("compute")
    rng = np.random.default_rng(sum(es) + sum(ks))
    env = (rng.random(int(np.prod(es))) < 0.4).astype(np.uint8)
    ker = (rng.random(int(np.prod(ks))) < 0.6).astype(np.uint8)
    ker[0] = 1
    spec = compute.CorrelationSpec(es, ks, (1, -2, 3), (0, 1, -1))
    _, _, want = oracle_c.correlate(False, es, ks, (1, -2, 3), (0, 1, -1), env, ker)
    padded = [e + k - 1 for e, k in zip(es, ks)]
    for precision in (compute.FP64, compute.FP32):
        got = compute.correlate_binary(spec, env, ker, context=gpu_ctx, precision=precision)
        assert isinstance(got, compute.CorrelationResult), got
        assert np.array_equal(got.values, want)
        assert list(got.padded_shape) == [_smooth(p) for p in padded]


def _smooth(n):
    """The smallest 2^a 3^b 5^c length >= n."""
    while True:
        m = n
        for p in (2, 3, 5):
            while m % p == 0:
                m //= p
        if m == 1:
            return n
        n += 1


def _open(ctx, box, catalog):
    assets, session_mod, synthetic = package("assets"), package("session"), package("synthetic")
    obj = assets.accept_stl(synthetic.cuboid_stl((10.0, 14.0, 20.0)))
    return session_mod.Session(obj, box, (0.0, 0.0, 0.0), 1.0, catalog, context=ctx)


@pytest.mark.parametrize("extent", [130, 150, 192])
def test_tuned_lengths_match_power_of_two(gpu_ctx, extent):
    geometry = package("geometry")
    catalog = geometry.cube_catalog()[:8]
    box = (float(extent - 2),) * 3  # the window adds a one-cell halo
    runs = {}
    for mode in ("tuned", "pow2"):
        if mode == "pow2":
            os.environ["SPK_FFT_LENGTHS"] = "pow2"
        try:
            s = _open(gpu_ctx, box, catalog)
            assert tuple(s.environment_shape) == (extent,) * 3
            pages = s.pages(range(len(catalog)))
            placed = [(p.orientation_index, p.translation, p.score) for p in s.greedy(4)]
            runs[mode] = (tuple(s.fft_shape), [[(c.translation, c.score) for c in p] for p in pages], placed)
            s.close()
        finally:
            os.environ.pop("SPK_FFT_LENGTHS", None)
    tuned, pow2 = runs["tuned"], runs["pow2"]
    assert pow2[0] == (256, 256, 256)
    assert tuned[1] == pow2[1] and tuned[2] == pow2[2]
    print(f"window {extent}^3: tuned lengths {tuned[0]}")


def test_odd_window_page_against_oracle(gpu_ctx, oracle_c):
    from oracle.bindings import oracle_page

    from scenes import scene

    pipeline = package("pipeline")
    sc = scene(11, shape=(70, 45, 39), kernel_shape=(9, 7, 8), blobs=10)
    prox, _ = oracle_c.build_proximity(sc["env_shape"], sc["occ"])
    page = pipeline.spectral_page(
        pipeline.PageScene(sc["env_first"], sc["env_shape"], sc["lattice"][:3], sc["lattice"][3], sc["cmin_z"],
                           sc["height"]),
        sc["occ"], sc["kernel_first"], sc["kernel_shape"], sc["kernel"], sc["max_z"], context=gpu_ctx)
    want = oracle_page(oracle_c, sc["env_first"], sc["env_shape"], sc["occ"], prox, sc["kernel_first"],
                       sc["kernel_shape"], sc["kernel"], sc["lattice"], sc["max_z"], sc["cmin_z"], sc["height"])
    assert [(p.translation, p.score) for p in page] == [(tuple(t), sc_) for t, sc_, _ in want]
