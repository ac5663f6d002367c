"""What the trained proposal network gains over the method without it.

On a held-out item in the 256^3 rounded container (512 orientations), each
of the first layouts of the exhaustive greedy fill is labelled with every
orientation's best exact score.  The trained network's top 32 must land
closer to the exhaustive choice than the untrained network's top 32.  The
untrained network is the same architecture and initialiser without training.
Closeness is measured two ways:
- regret: the best proposed score minus the best score overall;
- hit rate: the exhaustive choice is among the proposals.
"""

import os

import numpy as np
import pytest

from conftest import ROOT, package

pytestmark = pytest.mark.gpu
WEIGHTS = os.path.join(ROOT, "cpp-max-packer_b200", "weights", "proposal_rounded256.npz")
HELD_OUT_SEED = 7
STEPS = 4
K = 32


def test_trained_network_beats_untrained(gpu_ctx):
    assert os.path.exists(WEIGHTS), "trained proposal parameters are missing"
    proposal, train = package("proposal"), package("train_proposal")
    trained = proposal.Proposal(seed=7, context=gpu_ctx)
    trained.load(WEIGHTS)
    untrained = proposal.Proposal(seed=7, context=gpu_ctx)
    report = train.evaluate({"trained": trained, "untrained": untrained}, [HELD_OUT_SEED], STEPS, 512, K, gpu_ctx,
                            log=lambda *_: None)
    trained.close()
    untrained.close()
    t, u = report["trained"], report["untrained"]
    assert t["steps"] == STEPS and u["steps"] == STEPS
    assert t["mean_regret"] < u["mean_regret"], report
    assert t["hit_rate"] >= u["hit_rate"], report
    assert t["mean_regret"] <= report["random"]["mean_regret"], report
