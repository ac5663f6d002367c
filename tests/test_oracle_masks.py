"""The mask oracle on the host: its counts against the C oracle's full-range
correlation, and its masks against loops written straight from the
reference's rules (gap_fill.cpp:404-420 and :443-446)."""

import numpy as np

from oracle import masks


def _case(rng):
    es = rng.integers(1, 9, size=3)
    ks = rng.integers(1, 5, size=3)
    ef = rng.integers(-6, 6, size=3)
    kf = rng.integers(-6, 6, size=3)
    env = (rng.random(int(np.prod(es))) < rng.random()).astype(np.uint8)
    ker = (rng.random(int(np.prod(ks))) < 0.5).astype(np.uint8)
    ker[0] = 1
    return es, ks, ef, kf, env, ker


def test_direct_counts_match_the_c_oracle(oracle_c):
    rng = np.random.default_rng(40)
    for _ in range(20):
        es, ks, ef, kf, env, ker = _case(rng)
        tf, shape, counts = masks.direct_counts(es, ks, ef, kf, env, ker)
        ctf, cshape, want = oracle_c.correlate(False, es, ks, ef, kf, env, ker)
        assert list(tf) == list(ctf) and list(shape) == list(cshape)
        assert np.array_equal(counts, want.astype(np.int64))


def test_masks_follow_the_reference_rules():
    rng = np.random.default_rng(41)
    for _ in range(20):
        es, ks, ef, kf, env, ker = _case(rng)
        tf, shape, counts = masks.direct_counts(es, ks, ef, kf, env, ker)
        grid = counts.reshape(shape[2], shape[1], shape[0])
        # The legal box of gap_fill (first = window.first - kernel.first), and
        # a box that reaches past the range on every side.
        legal_first = [int(ef[a]) - int(kf[a]) for a in range(3)]
        legal_shape = [max(int(es[a]) - int(ks[a]) + 1, 0) for a in range(3)]
        wide_first = [tf[a] - 2 for a in range(3)]
        wide_shape = [shape[a] + 4 for a in range(3)]
        for first, bshape in ((legal_first, legal_shape), (wide_first, wide_shape), (tf, shape)):
            for want_zero in (True, False):
                got = masks.translation_mask(tf, shape, counts, first, bshape, want_zero)
                want = np.zeros(int(np.prod(bshape)), np.uint8)
                i = 0
                for z in range(bshape[2]):
                    for y in range(bshape[1]):
                        for x in range(bshape[0]):
                            o = (first[0] + x - tf[0], first[1] + y - tf[1], first[2] + z - tf[2])
                            inside = all(0 <= o[a] < shape[a] for a in range(3))
                            if inside:
                                c = grid[o[2], o[1], o[0]]
                                want[i] = (c == 0) if want_zero else (c != 0)
                            i += 1
                assert np.array_equal(got, want)


def test_box_far_outside_the_range_is_all_zero():
    counts = np.zeros(8)
    got = masks.translation_mask((0, 0, 0), (2, 2, 2), counts, (1 << 40, 0, 0), (3, 2, 1), True)
    assert got.shape == (6,) and not got.any()
