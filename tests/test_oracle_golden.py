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


def _pattern(shape, salt):
    # The deterministic binary fixture of correlation_tests.cpp:184-199:
    # a cell is set when (17x + 11y + 5z + 3xy + 7yz + 13xz + salt) mod 19 < 7,
    # and the first and last cells are always set.
    z, y, x = np.mgrid[0:shape[2], 0:shape[1], 0:shape[0]].astype(np.int64)
    cells = (((17 * x + 11 * y + 5 * z + 3 * x * y + 7 * y * z + 13 * x * z + salt) % 19) < 7).astype(np.uint8)
    cells = cells.reshape(-1)
    cells[0] = cells[-1] = 1
    return cells


def _checked_binary(oracle_c, es, ks, ef, kf, env, ker):
    # correlation_tests.cpp:68-110: the FFT oracle against the direct integer
    # oracle, whose kernel origin is kernel_first - environment_first.
    tf, shape, values = oracle_c.correlate(False, es, ks, ef, kf, env, ker)
    b = np.asarray(env, np.int64).reshape(es[2], es[1], es[0])
    k = np.asarray(ker, np.int64).reshape(ks[2], ks[1], ks[0])
    first, dshape, direct = oracle_c.correlate_int(b, k, [kf[a] - ef[a] for a in range(3)])
    assert list(shape) == [es[a] + ks[a] - 1 for a in range(3)] == list(dshape)
    assert [int(v) for v in tf] == [int(v) for v in first]
    assert np.array_equal(values, direct.astype(np.float64))


def test_proximity_matches_true_3d_direct_sum(oracle_c):
    # correlation_tests.cpp:329-347
    es, ks, ef, kf = (2, 2, 2), (2, 1, 2), (11, -7, 4), (-3, 5, 2)
    prox = np.array([0.0, 0.125, 0.25, 0.5, 0.75, 1.0, 0.375, 0.625])
    ker = np.array([1, 0, 1, 1], np.uint8)
    tf, shape, values = oracle_c.correlate(True, es, ks, ef, kf, prox, ker)
    e = prox.reshape(2, 2, 2)
    k = ker.reshape(2, 1, 2).astype(np.float64)
    want = np.zeros((shape[2], shape[1], shape[0]))
    for uz in range(shape[2]):
        for uy in range(shape[1]):
            for ux in range(shape[0]):
                s = 0.0
                for kz in range(ks[2]):
                    for ky in range(ks[1]):
                        for kx in range(ks[0]):
                            x, y, z = kx + ux - (ks[0] - 1), ky + uy - (ks[1] - 1), kz + uz - (ks[2] - 1)
                            if 0 <= x < es[0] and 0 <= y < es[1] and 0 <= z < es[2]:
                                s += e[z, y, x] * k[kz, ky, kx]
                want[uz, uy, ux] = s
    want = want.reshape(-1)
    assert np.all(np.abs(values - want) <= 1e-10 * np.maximum(1.0, np.abs(want)))


def _proper_cube_rotations():
    # The 24 proper rotations as (source axis, sign) per output axis: axis
    # permutations times sign patterns whose product with the permutation's
    # parity is +1 (correlation_tests.cpp:116-142).
    import itertools

    out = []
    for perm in itertools.permutations(range(3)):
        parity = 1 if sum(perm[i] > perm[j] for i in range(3) for j in range(i + 1, 3)) % 2 == 0 else -1
        for signs in itertools.product((-1, 1), repeat=3):
            if parity * signs[0] * signs[1] * signs[2] == 1:
                out.append((perm, signs))
    return out


def _rotate(shape, first, cells, perm, signs):
    # A cell at source world coordinate w lands at output coordinate
    # sign * w[source axis] (correlation_tests.cpp:149-182).
    rshape = [shape[perm[a]] for a in range(3)]
    rfirst = [first[perm[a]] if signs[a] > 0 else -(first[perm[a]] + shape[perm[a]] - 1) for a in range(3)]
    src = np.asarray(cells).reshape(shape[2], shape[1], shape[0])
    out = np.zeros((rshape[2], rshape[1], rshape[0]), np.uint8)
    for z in range(shape[2]):
        for y in range(shape[1]):
            for x in range(shape[0]):
                local = (x, y, z)
                o = [signs[a] * (first[perm[a]] + local[perm[a]]) - rfirst[a] for a in range(3)]
                out[o[2], o[1], o[0]] = src[z, y, x]
    return rshape, rfirst, out.reshape(-1)


def test_asymmetric_kernel_in_all_24_cube_rotations(oracle_c):
    # correlation_tests.cpp:438-465
    es, ef = (4, 5, 6), (8, -5, 11)
    env = _pattern(es, 2)
    ks, kf = (2, 3, 5), (-4, 2, -7)
    ker = _pattern(ks, 7)
    rotations = _proper_cube_rotations()
    assert len(rotations) == 24
    for perm, signs in rotations:
        rshape, rfirst, rcells = _rotate(ks, kf, ker, perm, signs)
        assert int(rcells.sum()) == int(ker.sum())
        _checked_binary(oracle_c, es, rshape, ef, rfirst, env, rcells)


@pytest.mark.parametrize("lengths", [(8, 6), (64, 64)])
def test_padded_lengths_13_and_127_on_every_axis(oracle_c, lengths):
    # correlation_tests.cpp:467-481 with qualify_padded_axis (:216-240):
    # full-range lengths 13 and 127 along one axis at a time.
    for axis in range(3):
        es, ks = [1, 1, 1], [1, 1, 1]
        es[axis], ks[axis] = lengths
        _checked_binary(oracle_c, es, ks, (6, -5, 9), (-3, 4, -7), _pattern(es, 3), _pattern(ks, 11))


def test_rotated_kernels_match_the_reference_build(oracle_c, oracle_ref):
    # The same 24 rotations through the reference's own correlate_binary_cpu.
    es, ef = (4, 5, 6), (8, -5, 11)
    env = _pattern(es, 2)
    ker = _pattern((2, 3, 5), 7)
    for perm, signs in _proper_cube_rotations():
        rshape, rfirst, rcells = _rotate((2, 3, 5), (-4, 2, -7), ker, perm, signs)
        want = oracle_ref.correlate(False, es, rshape, ef, rfirst, env, rcells)
        got = oracle_c.correlate(False, es, rshape, ef, rfirst, env, rcells)
        assert not isinstance(want, str), want
        assert list(got[0]) == list(want[0]) and list(got[1]) == list(want[1])
        assert np.array_equal(got[2], want[2])


def test_proximity_every_cell_of_empty_full_and_patterned_fields(oracle_c):
    # engine/pack_solver/tests/t009_tests.cpp:101-131: exp(-d/2) of the
    # Euclidean distance to the nearest occupied cell, by brute force over
    # every cell (0 where nothing is occupied), for 23 occupancy patterns.
    shape = (5, 3, 2)
    for pattern in range(23):
        occ = np.array([0 if pattern == 0 else 1 if pattern == 1 else int((i * 7 + pattern * 3) % 11 < 3)
                        for i in range(30)], np.uint8)
        values, _ = oracle_c.build_proximity(shape, occ)
        sites = [(i % 5, (i // 5) % 3, i // 15) for i in range(30) if occ[i]]
        for i in range(30):
            x, y, z = i % 5, (i // 5) % 3, i // 15
            d = min((math.sqrt((x - a) ** 2 + (y - b) ** 2 + (z - c) ** 2) for a, b, c in sites), default=math.inf)
            assert values[i] == (math.exp(-d / 2.0) if math.isfinite(d) else 0.0), (pattern, i)
