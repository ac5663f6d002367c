"""The oracle restatement pinned to the reference's golden vectors and to the
reference C++ compiled here (CPU only)."""

import math

import numpy as np
import pytest


def test_fsum_is_correctly_rounded(oracle_c):
    rng = np.random.default_rng(3)
    for _ in range(200):
        v = rng.standard_normal(rng.integers(1, 300)) * 10.0 ** rng.integers(-20, 20, size=1)
        assert oracle_c.fsum(v) == math.fsum(v)
    assert oracle_c.fsum([1e-16, 1.0, 1e16]) == math.fsum([1e-16, 1.0, 1e16])


def test_direct_integer_oracle_full_linear_range(oracle_c):
    # tests/native/integer_correlation_tests.cpp:11-33
    blocked = np.array([1, 2, 3, 4, 5, 6]).reshape(1, 2, 3)
    kernel = np.array([2, 0, 1, 3]).reshape(1, 2, 2)
    first, shape, values = oracle_c.correlate_int(blocked, kernel, (-1, 1, 0))
    assert list(first) == [0, -2, 0]
    assert list(shape) == [4, 3, 1]
    assert list(values) == [3, 7, 11, 3, 12, 21, 27, 12, 0, 8, 10, 12]


def test_direct_integer_oracle_all_axes(oracle_c):
    # tests/native/integer_correlation_tests.cpp:35-46
    blocked = np.array([1, 0, 2, 1, 3, 2, 0, 4, 1, 2, 0, 5]).reshape(2, 3, 2)
    kernel = np.array([2, 1, 0, 3]).reshape(2, 2, 1)
    first, shape, values = oracle_c.correlate_int(blocked, kernel, (0, 0, -1))
    assert list(shape) == [2, 4, 3]
    assert list(values) == [3, 0, 6, 3, 9, 6, 0, 0, 1, 12, 7, 7, 7, 19, 6, 4, 0, 4, 1, 10, 2, 9, 0, 10]


def test_binary_translation_range(oracle_c):
    # engine/pack_compute/tests/correlation_tests.cpp:292-308
    tf, shape, values = oracle_c.correlate(False, (3, 2, 1), (2, 2, 1), (4, -3, 0), (-1, 1, 0),
                                           [1, 0, 1, 0, 1, 1], [1, 0, 1, 1])
    assert list(tf) == [4, -5, 0] and list(shape) == [4, 3, 1]
    # Same numbers as the independent integer oracle with origin = kernel_first - env_first.
    _, _, direct = oracle_c.correlate_int(np.array([1, 0, 1, 0, 1, 1]).reshape(1, 2, 3),
                                          np.array([1, 0, 1, 1]).reshape(1, 2, 2), (-5, 4, 0))
    assert list(values) == list(direct)


def test_proximity_fractional_boundaries(oracle_c):
    # correlation_tests.cpp:310-327
    tf, shape, values = oracle_c.correlate(True, (2, 1, 1), (2, 1, 1), (9, 0, 0), (3, 0, 0), [0.5, 1.0], [1, 1])
    assert list(tf) == [5, 0, 0]
    assert np.allclose(values, [0.5, 1.5, 1.0], atol=0.25)


def test_true_3d_asymmetric_range(oracle_c):
    # correlation_tests.cpp:416-437
    env = [1, 0, 1, 0, 1, 1, 0, 1, 0, 1, 1, 0]
    tf, shape, _ = oracle_c.correlate(False, (2, 3, 2), (1, 2, 2), (7, -4, 9), (-3, 5, -2), env, [1, 0, 1, 1])
    assert list(tf) == [10, -10, 10]
    assert [tf[a] + shape[a] - 1 for a in range(3)] == [11, -7, 12]


def _random_case(rng, proximity):
    es = rng.integers(1, 9, size=3)
    ks = rng.integers(1, 6, size=3)
    ef = rng.integers(-20, 20, size=3)
    kf = rng.integers(-20, 20, size=3)
    env = rng.random(int(np.prod(es))) if proximity else (rng.random(int(np.prod(es))) < 0.5).astype(np.uint8)
    ker = (rng.random(int(np.prod(ks))) < 0.6).astype(np.uint8)
    return es, ks, ef, kf, env, ker


@pytest.mark.parametrize("proximity", [False, True])
def test_oracle_matches_reference_correlation(oracle_c, oracle_ref, proximity):
    rng = np.random.default_rng(11 + proximity)
    for _ in range(40):
        es, ks, ef, kf, env, ker = _random_case(rng, proximity)
        want = oracle_ref.correlate(proximity, es, ks, ef, kf, env, ker)
        got = oracle_c.correlate(proximity, es, ks, ef, kf, env, ker)
        if isinstance(want, str):  # the reference fails closed (e.g. empty kernel mass)
            continue
        assert list(got[0]) == list(want[0]) and list(got[1]) == list(want[1])
        if proximity:
            assert np.allclose(got[2], want[2], rtol=0, atol=1e-10 * max(1.0, np.abs(want[2]).max()))
        else:
            assert np.array_equal(got[2], want[2])


def test_oracle_proximity_field_bit_exact_with_reference(oracle_c, oracle_ref):
    rng = np.random.default_rng(5)
    for shape in [(1, 1, 1), (5, 4, 3), (13, 7, 9), (20, 20, 20)]:
        for density in (0.0, 0.02, 0.3):
            occ = (rng.random(int(np.prod(shape))) < density).astype(np.uint8)
            want = oracle_ref.build_proximity(shape, occ)
            got, _ = oracle_c.build_proximity(shape, occ)
            assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
