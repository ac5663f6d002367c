"""Independent jobs filled concurrently (spk_jobs_greedy) give exactly the
placements each job gives alone: uneven windows (66^3, 128^3, 40^3-class),
cuboid and blob items, exhaustive and proposed greedy."""

import numpy as np
import pytest

from conftest import package
from oracle import proposal_net

pytestmark = pytest.mark.gpu


def _jobs():
    workloads, synthetic, assets, geometry = (package("workloads"), package("synthetic"), package("assets"),
                                              package("geometry"))
    small_blob = assets.accept_stl(synthetic.blob_stl(5, level=3, base_mesh="icosahedron", radius_range=(4.0, 6.0)))
    return [
        (workloads.box64_cuboid_cube24(), 6, False),
        (workloads.box63_blob_hopf96(), 3, False),
        (workloads.Workload("box40_blob_hopf32", small_blob, (40.0, 36.0, 30.0), (0.0, 0.0, 0.0), 1.0,
                            geometry.hopf_catalog(32, 5)), 5, True),
    ]


def _open(wl, compute, session_mod):
    ctx = compute.Context(0)
    return ctx, session_mod.Session(wl.obj, wl.container, wl.origin, wl.pitch, wl.catalog, context=ctx)


def test_concurrent_jobs_match_each_job_alone():
    compute, session_mod, proposal = package("compute"), package("session"), package("proposal")
    jobs = _jobs()
    flat = proposal_net.he_parameters(9).astype(np.float32)
    alone = []
    for wl, steps, learned in jobs:
        ctx, s = _open(wl, compute, session_mod)
        if learned:
            net = proposal.Proposal(context=ctx)
            net.set_parameters(flat)
            placed, fb = proposal.greedy_proposed(s, net, 4, steps)
            net.close()
        else:
            placed, fb = s.greedy(steps), 0
        alone.append(([(p.orientation_index, p.translation, p.score) for p in placed], fb))
        s.close()
        ctx.close()
    contexts, sessions, nets, spec = [], [], [], []
    for wl, steps, learned in jobs:
        ctx, s = _open(wl, compute, session_mod)
        net = None
        if learned:
            net = proposal.Proposal(context=ctx)
            net.set_parameters(flat)
            nets.append(net)
        contexts.append(ctx)
        sessions.append(s)
        spec.append((s, net, 4, steps))
    together = session_mod.run_jobs(spec)
    for (placed, fb), (want, want_fb) in zip(together, alone):
        assert [(p.orientation_index, p.translation, p.score) for p in placed] == want
        assert fb == want_fb
    for n in nets:
        n.close()
    for s, ctx in zip(sessions, contexts):
        s.close()
        ctx.close()
