"""GPU spectral pages against the oracle page restatement (exact parity)."""

import numpy as np
import pytest

from conftest import package
from oracle.bindings import oracle_page
from scenes import scene

pytestmark = pytest.mark.gpu


def _gpu_page(sc, orientation=0, cursor=None, ctx=None, report=None):
    pl = package("pipeline")
    s = pl.PageScene(sc["env_first"], sc["env_shape"], sc["lattice"][:3], sc["lattice"][3], sc["cmin_z"],
                     sc["height"])
    return pl.spectral_page(s, sc["occ"], sc["kernel_first"], sc["kernel_shape"], sc["kernel"], sc["max_z"],
                            orientation, cursor, context=ctx, report=report)


def _oracle_page(oracle_c, sc, orientation=0, cursor=None):
    prox, _ = oracle_c.build_proximity(sc["env_shape"], sc["occ"])
    return oracle_page(oracle_c, sc["env_first"], sc["env_shape"], sc["occ"], prox, sc["kernel_first"],
                       sc["kernel_shape"], sc["kernel"], sc["lattice"], sc["max_z"], sc["cmin_z"], sc["height"],
                       orientation, cursor)


def _same(gpu, ora):
    assert len(gpu) == len(ora)
    for g, (t, score, o) in zip(gpu, ora):
        assert g.translation == tuple(t)
        assert g.orientation_index == o
        assert g.score == score  # bit-identical: both are the correctly rounded exact sum
        assert g.direct_zero_overlap and g.binary_overlap == 0.0


@pytest.mark.parametrize("seed", range(6))
def test_blob_pages_match_oracle(gpu_ctx, oracle_c, seed):
    sc = scene(seed)
    rep = {}
    gpu = _gpu_page(sc, orientation=seed, ctx=gpu_ctx, report=rep)
    _same(gpu, _oracle_page(oracle_c, sc, orientation=seed))
    assert rep["max_integer_residual"] < 0.25


def test_cursor_pages_chain(gpu_ctx, oracle_c):
    sc = scene(42)
    cursor = None
    for _ in range(4):
        gpu = _gpu_page(sc, orientation=3, cursor=cursor, ctx=gpu_ctx)
        ora = _oracle_page(oracle_c, sc, orientation=3,
                           cursor=None if cursor is None else (cursor.translation, cursor.score, 3))
        _same(gpu, ora)
        if not gpu:
            break
        cursor = gpu[-1]


def test_symmetric_ties_take_the_threshold_path(gpu_ctx, oracle_c):
    # A cuboid in an empty box: many exactly equal scores (ties resolved by z, y, x).
    sc = scene(7, shape=(30, 30, 24), kernel_shape=(6, 8, 5), blobs=0, cuboid=True)
    rep = {}
    gpu = _gpu_page(sc, ctx=gpu_ctx, report=rep)
    _same(gpu, _oracle_page(oracle_c, sc))


def test_kernel_wider_than_environment_is_an_empty_page(gpu_ctx):
    sc = scene(1, shape=(12, 12, 12), kernel_shape=(13, 5, 5))
    assert _gpu_page(sc, ctx=gpu_ctx) == []


def test_full_layout_has_no_candidates(gpu_ctx):
    sc = scene(2)
    sc["occ"] = np.ones_like(sc["occ"])
    assert _gpu_page(sc, ctx=gpu_ctx) == []


@pytest.mark.parametrize("seed", [11, 12])
def test_pages_on_a_256_grid_match_oracle(gpu_ctx, oracle_c, seed):
    # E in (128, 256] on every axis selects the 256^3 register-FFT kernels.
    sc = scene(seed, shape=(200, 180, 160), kernel_shape=(9, 7, 8), blobs=40)
    rep = {}
    gpu = _gpu_page(sc, orientation=1, ctx=gpu_ctx, report=rep)
    _same(gpu, _oracle_page(oracle_c, sc, orientation=1))
    assert rep["max_integer_residual"] < 0.25
