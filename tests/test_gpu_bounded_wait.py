"""The expiry path of the library's bounded device waits.

The tcgen05 convolutions wait on mbarriers with a bounded poll count and
report SPK_DEVICE_WAIT_LIMIT when a wait runs out. spk_check_bounded_wait
makes such a wait run out: an mbarrier that nothing arrives at, polled a
thousand times. No GPU fault or hang is involved. The status must come back,
and the same context must then run a proposal forward and a correlation
correctly.
"""

import time

import numpy as np
import pytest

from conftest import package

pytestmark = pytest.mark.gpu


def test_expired_wait_reports_its_status_and_the_context_stays_usable(gpu_ctx):
    lib_mod, compute, proposal = package("_lib"), package("compute"), package("proposal")
    lib = lib_mod.lib()
    t0 = time.perf_counter()
    status = lib.spk_check_bounded_wait(gpu_ctx.handle, 1000)
    assert time.perf_counter() - t0 < 10.0
    assert status == 24 and lib_mod.status_code(status) == "SPK_DEVICE_WAIT_LIMIT"
    assert lib.spk_check_bounded_wait(gpu_ctx.handle, 0) != 0  # zero polls: rejected before any launch
    # The context still works: a proposal forward and a binary correlation.
    net = proposal.Proposal(seed=3, context=gpu_ctx)
    x = np.random.default_rng(0).random((2, 32, 32, 32, 2)).astype(np.float32)
    pred = net.forward(x)
    assert pred.shape[0] == 2 and np.all(np.isfinite(pred))
    net.close()
    spec = compute.CorrelationSpec((4, 4, 4), (2, 2, 2), (0, 0, 0), (0, 0, 0))
    env, ker = np.zeros(64, np.uint8), np.ones(8, np.uint8)
    env[0] = 1
    out = compute.correlate_binary(spec, env, ker, context=gpu_ctx)
    assert not isinstance(out, compute.CorrelationFailure)
    values = np.asarray(out.values).reshape(5, 5, 5)
    assert values[1, 1, 1] == 1.0 and values.sum() == 8.0
