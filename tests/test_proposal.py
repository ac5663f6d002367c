"""Proposal network: the numpy oracle pinned by finite differences (CPU), the
tensor-core forward and backward kernels against the oracle (GPU), training,
and the session's proposal path (GPU)."""

import numpy as np
import pytest

from conftest import package
from oracle import proposal_net as oracle


def _inputs(rng, batch, side=32):
    crop = rng.uniform(0, 1, (batch, side, side, side)) * (rng.uniform(0, 1, (batch, side, side, side)) < 0.4)
    zz, yy, xx = np.mgrid[0:side, 0:side, 0:side]
    items = []
    for _ in range(batch):
        r = rng.uniform(3, 9, 3)
        c = r + rng.uniform(0, 2, 3)
        items.append(((((xx - c[0]) / r[0]) ** 2 + ((yy - c[1]) / r[1]) ** 2 + ((zz - c[2]) / r[2]) ** 2) < 1)
                     .astype(np.float64))
    return np.stack([crop, np.stack(items)], axis=-1).astype(np.float32)


def test_parameter_layout_matches_oracle():
    proposal = package("proposal")
    count = sum(int(np.prod(s)) for _, s in proposal.parameter_layout())
    assert count == len(oracle.he_parameters(0))
    assert count == sum(cout * 27 * cin + cout for cin, cout, _ in oracle.LAYERS) + 65


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(3)
    flat = oracle.he_parameters(5, scale_head=0.5)
    x = _inputs(rng, 2, side=8).astype(np.float64)
    labels = np.array([0.3, -0.2])
    loss, grad = oracle.gradients(flat, x, labels, rounding=False)
    sizes = [cout * 27 * cin for cin, cout, _ in oracle.LAYERS]
    offsets = np.cumsum([0] + [s + c for s, (_, c, _) in zip(sizes, oracle.LAYERS)])
    picks = []
    for i, off in enumerate(offsets[:-1]):
        picks += list(off + rng.integers(0, sizes[i], 4))  # weights of every layer
        picks.append(off + sizes[i])                      # a bias of every layer
    picks += [offsets[-1] + 3, offsets[-1] + 64]          # head weight and bias
    h = 1e-6
    for p in picks:
        up, dn = flat.copy(), flat.copy()
        up[p] += h
        dn[p] -= h
        fd = (oracle.gradients(up, x, labels, rounding=False)[0] - oracle.gradients(dn, x, labels, rounding=False)[0])
        fd /= 2 * h
        assert abs(fd - grad[p]) <= 1e-6 + 1e-4 * abs(fd), (p, fd, grad[p])


def test_bf16_rounding_ties_to_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -2.5], np.float32)
    assert list(oracle.bf16(v)) == [1.0, 1.0, 1.0 + 2 ** -6, 1.0, -2.5]


@pytest.fixture(scope="module")
def net(gpu_ctx):
    n = package("proposal").Proposal(seed=11, context=gpu_ctx)
    yield n
    n.close()


def _set_oracle_parameters(net, seed):
    flat = oracle.he_parameters(seed).astype(np.float32)
    net.set_parameters(flat)
    return flat.astype(np.float64)


@pytest.mark.gpu
def test_forward_matches_oracle(net):
    flat = _set_oracle_parameters(net, 1)
    x = _inputs(np.random.default_rng(1), 3)
    got = net.forward(x)
    want, _, _ = oracle.forward(flat, x)
    # BF16 activations: the device's FP32 sums may round an activation one BF16
    # step away from the oracle's exact sums; the bound covers a few such steps.
    assert np.all(np.isfinite(got))
    assert np.abs(got - want).max() <= 1e-2 * np.abs(want).max() + 1e-3, (got, want)


@pytest.mark.gpu
def test_gradients_match_oracle(net):
    flat = _set_oracle_parameters(net, 2)
    rng = np.random.default_rng(2)
    x = _inputs(rng, 4)
    labels = rng.uniform(-0.3, 0.7, 4).astype(np.float32)
    loss, grad = net.gradients(x, labels)
    want_loss, want = oracle.gradients(flat, x, labels)
    assert abs(loss - want_loss) <= 2e-2 * abs(want_loss) + 1e-5
    off = 0
    for name, shape in package("proposal").parameter_layout():
        n = int(np.prod(shape))
        g, w = grad[off:off + n].astype(np.float64), want[off:off + n]
        off += n
        scale = np.linalg.norm(w)
        # Relative L2 error of each parameter block, BF16 storage of the
        # activations and pre-activation gradients included.
        assert np.linalg.norm(g - w) <= 3e-2 * scale + 1e-7, (name, np.linalg.norm(g - w), scale)


@pytest.mark.gpu
def test_forward_is_batch_independent(net):
    _set_oracle_parameters(net, 3)
    x = _inputs(np.random.default_rng(3), 5)
    whole = net.forward(x)
    parts = np.concatenate([net.forward(x[:2]), net.forward(x[2:])])
    assert np.array_equal(whole, parts)


@pytest.mark.gpu
def test_training_reduces_loss(gpu_ctx):
    proposal = package("proposal")
    net = proposal.Proposal(seed=4, context=gpu_ctx)
    rng = np.random.default_rng(4)
    crops = _inputs(rng, 8)[..., 0]
    items = _inputs(rng, 16)[..., 1]
    # Label: how high the item reaches (a pure function of the item channel).
    height = np.array([np.nonzero(it.any(axis=(1, 2)))[0].max() for it in items]) / 32.0
    sc = np.repeat(np.arange(8), 16).astype(np.uint32)
    si = np.tile(np.arange(16), 8).astype(np.uint32)
    data = proposal.ProposalDataset(crops, items, sc, si, height[si].astype(np.float32))
    losses = net.train(data, batch=32, steps=150, learning_rate=2e-3, seed=1)
    assert np.all(np.isfinite(losses))
    assert losses[-10:].mean() < 0.25 * losses[:10].mean(), (losses[:10].mean(), losses[-10:].mean())
    net.close()


def _small_session(gpu_ctx):
    workloads, session_mod = package("workloads"), package("session")
    wl = workloads.box64_cuboid_cube24()
    return session_mod.Session(wl.obj, wl.container, wl.origin, wl.pitch, wl.catalog, context=gpu_ctx), wl


@pytest.mark.gpu
def test_session_features_and_proposal(gpu_ctx, net):
    proposal = package("proposal")
    s, wl = _small_session(gpu_ctx)
    crop, items = proposal.session_features(s)
    assert crop.shape == (32, 32, 32) and items.shape == (len(wl.catalog), 32, 32, 32)
    occ = s.field("occupancy").reshape(tuple(reversed(s.environment_shape)))
    # 66^3 window pooled by 3: cell (0,0,0) covers the halo corner block.
    assert crop[0, 0, 0] == pytest.approx(occ[:3, :3, :3].mean(), abs=2 ** -8)
    assert np.all((items >= 0) & (items <= 1)) and items.sum() > 0
    best, pred = proposal.propose(s, net, 5)
    assert len(set(best.tolist())) == 5
    assert np.all(pred[best].max() <= np.delete(pred, best)) if len(pred) > 5 else True
    s.close()


@pytest.mark.gpu
def test_proposed_greedy_with_every_orientation_is_the_exhaustive_greedy(gpu_ctx, net):
    proposal = package("proposal")
    s, wl = _small_session(gpu_ctx)
    want = s.greedy(6)
    s.close()
    s, wl = _small_session(gpu_ctx)
    got, fallbacks = proposal.greedy_proposed(s, net, len(wl.catalog), 6)
    assert fallbacks == 0
    assert [(p.orientation_index, p.translation, p.score) for p in got] == \
        [(p.orientation_index, p.translation, p.score) for p in want]
    s.close()


@pytest.mark.gpu
def test_margin_greedy_reduces_to_the_fixed_and_exhaustive_greedies(gpu_ctx, net):
    # A zero margin with k_max = k_min pages exactly the k_min best, as the
    # proposed greedy with k = k_min; k_min = every orientation is the
    # exhaustive greedy.
    proposal = package("proposal")
    s, wl = _small_session(gpu_ctx)
    want, _ = proposal.greedy_proposed(s, net, 5, 6)
    s.close()
    s, wl = _small_session(gpu_ctx)
    got, fallbacks, paged = proposal.greedy_proposed_margin(s, net, 5, 5, 0.0, 6)
    assert [(p.orientation_index, p.translation, p.score) for p in got] == \
        [(p.orientation_index, p.translation, p.score) for p in want]
    assert paged == 5 * len(got)
    s.close()
    s, wl = _small_session(gpu_ctx)
    exhaustive = s.greedy(6)
    s.close()
    s, wl = _small_session(gpu_ctx)
    O = len(wl.catalog)
    got, fallbacks, paged = proposal.greedy_proposed_margin(s, net, O, O, 0.5, 6)
    assert fallbacks == 0 and paged == O * len(got)
    assert [(p.orientation_index, p.translation, p.score) for p in got] == \
        [(p.orientation_index, p.translation, p.score) for p in exhaustive]
    s.close()


@pytest.mark.gpu
def test_proposed_greedy_places_exact_copies(gpu_ctx, net):
    proposal = package("proposal")
    s, wl = _small_session(gpu_ctx)
    got, fallbacks = proposal.greedy_proposed(s, net, 3, 5)
    assert len(got) == 5
    best, _ = proposal.propose(s, net, 3)
    assert len(best) == 3
    s.close()


@pytest.mark.gpu
def test_session_predictions_match_the_plain_forward(gpu_ctx, net):
    # The session path caches the first layer's item-channel sums; it must
    # score exactly what the plain forward pass scores on the same inputs, on
    # later layouts, and again after the parameters change.
    proposal = package("proposal")
    _set_oracle_parameters(net, 4)
    s, wl = _small_session(gpu_ctx)
    _, items = proposal.session_features(s)
    for step in range(3):
        if step == 2:
            _set_oracle_parameters(net, 5)
        crop = proposal.session_crop(s)
        _, pred = proposal.propose(s, net, 3)
        want = net.forward(np.stack([np.broadcast_to(crop, items.shape), items], axis=-1))
        assert np.abs(pred - want).max() <= 2e-3 * np.abs(want).max() + 1e-5, (step, pred, want)
        s.greedy(1)
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("workload", ["box64_cuboid_cube24", "rounded256_blob_hopf512"])
def test_corner_box_trunk_equals_the_full_split_forward(gpu_ctx, net, workload):
    # The session path runs every layer once on the layout alone and, per
    # orientation, only over the corner box its item reaches, and between
    # calls recomputes only the voxels a layout change reaches.  Its
    # predictions must equal, value for value, the full split forward's
    # (SPK_PROPOSAL_TRUNK=full, on a second network with the same
    # parameters): over successive placements, after a removal, on an
    # unchanged layout, and after a parameter change.
    import os

    proposal, workloads, session_mod = package("proposal"), package("workloads"), package("session")
    full = proposal.Proposal(seed=11, context=gpu_ctx)
    for n in (net, full):
        _set_oracle_parameters(n, 6)
    kwargs = {"orientations": 24} if workload.startswith("rounded256") else {}
    wl = getattr(workloads, workload)(**kwargs)
    s = session_mod.Session(wl.obj, wl.container, wl.origin, wl.pitch, wl.catalog, context=gpu_ctx)
    for step in range(6):
        if step == 3:
            s.remove_last()  # the layout goes back: a change the trunk must see
        if step == 5:
            for n in (net, full):
                _set_oracle_parameters(n, 7)
        best, pred = proposal.propose(s, net, 4)
        again_best, again = proposal.propose(s, net, 4)  # unchanged layout
        os.environ["SPK_PROPOSAL_TRUNK"] = "full"
        try:
            best_full, pred_full = proposal.propose(s, full, 4)
        finally:
            os.environ.pop("SPK_PROPOSAL_TRUNK", None)
        assert np.array_equal(pred, pred_full), (step, np.abs(pred - pred_full).max())
        assert np.array_equal(again, pred) and np.array_equal(best, best_full)
        if step != 2:
            s.greedy(1)
    s.close()
    full.close()
