"""The host mirror's own checks, which come before any device work and so run
without a GPU: extents, then cell counts, with the reference's codes and in
its order (correlation.cpp:276-312)."""

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
