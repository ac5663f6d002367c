"""The multi-job configuration at a reduced size: independent jobs of uneven
windows (64..192 cells per axis), blob and cuboid items and 96..512
orientations, filled concurrently by spk_jobs_greedy with the learned
proposal on (cpp-max-packer_b200/multi_job.py builds the jobs).

Every placement goes through the reference's own geometry::validate_incremental
as the job's try_pose gate (the reference build, oracle/_ref): none may be
rejected.  The windows' transform lengths come from the autotuner, so most
jobs run on non-power-of-two grids.
"""

import numpy as np
import pytest

from conftest import package

pytestmark = pytest.mark.gpu


@pytest.mark.timeout(1200)
def test_multi_job_placements_pass_the_reference_validator(oracle_ref):
    compute, proposal, session_mod, geometry = (package("compute"), package("proposal"), package("session"),
                                                package("geometry"))
    multi = package("multi_job")
    specs = multi.job_specs(8, seed=11, max_orientations=160)
    weights = __import__("os").path.join(multi.HERE, "weights", "proposal_rounded256.npz")
    jobs, refs, offered = [], [], []
    for spec in specs:
        ctx = compute.Context(0)
        s, obj, box = multi.open_job(spec, ctx)
        net = proposal.Proposal(context=ctx)
        net.load(weights)
        catalog = oracle_ref.catalog(4, geometry.hopf_quaternions(spec.orientations, spec.catalog_seed))
        assert np.array_equal(catalog, s.catalog)
        ref_session = oracle_ref.session(oracle_ref.asset(multi.item_stl(spec)), box, 0.0, 0.0, (0.0, 0.0, 0.0), 1.0,
                                         catalog)
        seen = []

        def validate(orientation, t, pose_mm, q, ref_session=ref_session, seen=seen):
            seen.append((orientation, t))
            return ref_session.place(orientation, t)

        s.set_validator(validate)
        jobs.append((ctx, s, net))
        refs.append(ref_session)
        offered.append(seen)
    results = session_mod.run_jobs([(s, net, 32, 3) for _, s, net in jobs])
    total = 0
    for (placed, _), (ctx, s, net), seen in zip(results, jobs, offered):
        validated, rejected = s.validation_counts()
        assert rejected == 0 and validated == len(placed) == len(seen)
        total += len(placed)
    assert total >= 8
    non_pow2 = sum(any(L & (L - 1) for L in s.fft_shape) for _, s, _ in jobs)
    print(f"{len(jobs)} jobs, {total} placements validated by the reference, 0 rejected; "
          f"{non_pow2} jobs on non-power-of-two grids")
    for ctx, s, net in jobs:
        s.set_validator(None)
        net.close()
        s.close()
        ctx.close()
