"""Host-side logic that runs without a GPU.  It covers two things:
- the mirror's own checks, which come before any device work: extents, then
  cell counts, with the reference's codes and in its order
  (correlation.cpp:263-312);
- the proposal trainer's label definition, layout schedule and dataset merge.
"""

import numpy as np

from conftest import package


def test_field_checks_come_before_the_device():
    compute = package("compute")
    spec = compute.CorrelationSpec((4, 3, 2), (2, 2, 2), (0, 0, 0), (1, 1, 1))
    env, ker = np.zeros(24, np.uint8), np.ones(8, np.uint8)
    calls = (
        lambda s, e, k: compute.correlate_binary(s, e, k),
        lambda s, e, k: compute.correlate_proximity(s, e.astype(np.float64), k),
        lambda s, e, k: compute.correlate_binary_mask(s, e, k, (0, 0, 0), (2, 2, 2)),
    )
    for call in calls:
        short = call(spec, env[:-1], ker)
        assert isinstance(short, compute.CorrelationFailure) and short.code == "CORRELATION_INVALID_FIELD"
        zero = compute.CorrelationSpec((4, 0, 2), (2, 2, 2))
        empty = call(zero, env, ker)
        assert isinstance(empty, compute.CorrelationFailure) and empty.code == "CORRELATION_SHAPE_OVERFLOW"
        assert empty.message == "Correlation extents must be positive and representable."


def test_an_interruption_wins_over_a_bad_field():
    compute = package("compute")
    spec = compute.CorrelationSpec((4, 3, 2), (2, 2, 2))
    control = compute.OperationControl()
    control.request_stop()
    r = compute.correlate_binary(spec, np.zeros(23, np.uint8), np.ones(8, np.uint8), control=control)
    assert r.code == "OPERATION_CANCELLED" and r.message == "Correlation interrupted."
    r = compute.correlate_binary(spec, np.zeros(23, np.uint8), np.ones(8, np.uint8),
                                 control=compute.OperationControl(deadline_ns=1))
    assert r.code == "DEADLINE_EXCEEDED"


def test_proposal_labels_and_layout_schedule():
    # Labels: each orientation's gap to the layout's best exact score, clipped
    # at the cap and scaled to [0, 1]; no admissible copy labels 1; a layout
    # where nothing is admissible gives no labels.
    train = package("train_proposal")
    best = np.array([-0.30, -0.29, np.inf, 0.10, -0.30])
    y = train.labels_from(best, 0.25)
    assert y.dtype == np.float32
    assert np.allclose(y, [0.0, 0.04, 1.0, 1.0, 0.0], atol=1e-6)
    assert train.labels_from(np.full(3, np.inf), 0.25) is None
    # Every step up to `dense`, then every `stride`-th.
    assert train.labelled_steps(3, 10, 35) == [0, 1, 2, 3, 13, 23, 33]


def test_policy_layouts_merge_with_reindexed_crops():
    # Policy layouts index their crops from 0; their items already start at
    # the base dataset's item count (generate_policy's item_base_count).
    train, proposal = package("train_proposal"), package("proposal")
    base = proposal.ProposalDataset(np.zeros((2, 4)), np.zeros((3, 4)), np.array([0, 1], np.uint32),
                                    np.array([2, 0], np.uint32), np.array([0.1, 0.2], np.float32))
    extra = ([np.ones(4)], [np.ones((2, 4))], [np.full(2, 0, np.uint32)], [3 + np.arange(2, dtype=np.uint32)],
             [np.array([0.3, 0.4], np.float32)])
    merged = train.merge_datasets(base, *extra)
    assert merged.crops.shape == (3, 4) and merged.items.shape == (5, 4)
    assert merged.sample_crop.tolist() == [0, 1, 2, 2]
    assert merged.sample_item.tolist() == [2, 0, 3, 4]
    assert np.allclose(merged.sample_label, [0.1, 0.2, 0.3, 0.4])
    assert train.merge_datasets(base, [], [], [], [], []) is base


def test_page_arrays_convert_like_the_per_element_reader():
    # candidates_from_c reads a CandidateC array column by column; it must
    # give the values, types and hashes of RankedCandidate.from_c.
    pipeline = package("pipeline")
    rng = np.random.default_rng(5)
    pages = (pipeline.CandidateC * (8 * pipeline.PAGE_SIZE))()
    for c in pages:
        for a in range(3):
            c.translation[a] = int(rng.integers(-2**40, 2**40))
        c.score = float(rng.normal())
        c.direct_zero_overlap = int(rng.integers(0, 2))
        c.orientation_index = int(rng.integers(0, 2**63))
        c.binary_overlap = float(rng.integers(0, 100))
    counts = [0, 1, 32, 17, 5, 32, 2, 9]
    want = [[pipeline.RankedCandidate.from_c(pages[i * pipeline.PAGE_SIZE + k]) for k in range(n)]
            for i, n in enumerate(counts)]
    got = pipeline.candidates_from_c(pages, counts, pipeline.PAGE_SIZE)
    assert got == want
    for page_got, page_want in zip(got, want):
        for a, b in zip(page_got, page_want):
            assert hash(a) == hash(b)
            assert type(a.translation[0]) is int and type(a.score) is float
            assert type(a.direct_zero_overlap) is bool and type(a.orientation_index) is int
