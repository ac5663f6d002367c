"""bench.py's multi-rank plumbing on the host: two gloo ranks.

Under torchrun each rank packs its own seeded job, so the only exchange is
the timing reduction: the slowest rank's device time and the sum of all
ranks' placements.  The reference arm runs on rank 0 alone; other ranks
return without work or output.
"""

import datetime
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, times, placed, results):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as tdist

    import bench

    tdist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        results.put((rank, bench.max_over_ranks(times[rank], placed[rank], world)))
        tdist.barrier()
    finally:
        tdist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_ranks_reduce_to_slowest_time_and_total_placements():
    import torch.multiprocessing as mp

    world, times, placed = 2, [12.5, 31.25], [7, 9]
    ctx = mp.get_context("spawn")
    results = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, times, placed, results)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(results.get(timeout=150) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == {0: (31.25, 16.0), 1: (31.25, 16.0)}


def test_single_rank_needs_no_process_group():
    import bench

    assert bench.max_over_ranks(4.0, 3, 1) == (4.0, 3.0)


def test_reference_arm_runs_on_rank_zero_only(capsys):
    import argparse

    import bench

    args = argparse.Namespace(workload="rounded256_blob_hopf512", orientations=0, warmup=3, steps=1)
    assert bench.run_reference(args, rank=1, world=2) is None
    assert capsys.readouterr().out == ""
