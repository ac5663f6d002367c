"""The multi-job configuration: many independent packing jobs of uneven
window sizes filled at once on one GPU.

    python cpp-max-packer_b200/multi_job.py [--jobs 64] [--steps 8] [--seed 5] [--k 32]

Jobs are seeded stand-ins with the configuration's shapes:
- a box container whose window is uniform in 64..192 cells per axis (1 mm
  pitch; the window adds a one-cell halo);
- an item from the blob generator with 2,048, 5,120 or 8,192 triangles
  (octahedron level 4, icosahedron level 4, octahedron level 5; radius
  4-10 mm), or a seeded cuboid (12 triangles);
- a catalog of 96..512 seeded SO(3) orientations;
- the learned proposal on (top k, exhaustive fallback), with the committed
  network parameters.

Every placement is an exact candidate (a zero exact overlap recount and the
exact FP64 score); the validation of each placement through the reference's
own validator is covered by tests/test_gpu_multi_job.py.

Each job has its own context and session.  spk_jobs_greedy runs every job
on its own host thread and stream, so the device interleaves kernels of
different jobs.  Printed: the jobs' windows and chosen transform lengths,
placements per job, and the wall time and placements/s of the concurrent
fill against the same jobs filled one after another.
"""

from __future__ import annotations

import argparse
import dataclasses
import importlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pkg(name):
    return importlib.import_module("cpp-max-packer_b200." + name)


@dataclasses.dataclass
class JobSpec:
    name: str
    window: tuple  # cells per axis, halo included
    item: str  # "blob2048", "blob5120", "blob8192" or "cuboid"
    item_seed: int
    orientations: int
    catalog_seed: int


def job_specs(count: int, seed: int, max_orientations: int = 512) -> list:
    """Seeded jobs with the multi-job configuration's shapes."""
    rng = np.random.default_rng(seed)
    items = ["blob2048", "blob5120", "blob8192", "cuboid"]
    out = []
    for j in range(count):
        window = tuple(int(v) for v in rng.integers(64, 193, size=3))
        item = items[int(rng.integers(0, len(items)))]
        orientations = int(min(rng.integers(96, 513), max_orientations))
        out.append(JobSpec(f"job{j}", window, item, int(rng.integers(0, 1 << 20)), orientations,
                           int(rng.integers(0, 1 << 20))))
    return out


def item_stl(spec: JobSpec) -> bytes:
    synthetic = pkg("synthetic")
    if spec.item == "cuboid":
        rng = np.random.default_rng(spec.item_seed)
        return synthetic.cuboid_stl(tuple(float(v) for v in rng.uniform(6.0, 16.0, size=3)))
    level, base = {"blob2048": (4, "octahedron"), "blob5120": (4, "icosahedron"),
                   "blob8192": (5, "octahedron")}[spec.item]
    return synthetic.blob_stl(spec.item_seed, level=level, base_mesh=base, radius_range=(4.0, 10.0))


def open_job(spec: JobSpec, context):
    """(session, object mesh, box) for a job on `context`."""
    assets, geometry, session_mod = pkg("assets"), pkg("geometry"), pkg("session")
    obj = assets.accept_stl(item_stl(spec))
    box = tuple(float(v - 2) for v in spec.window)
    catalog = geometry.hopf_catalog(spec.orientations, spec.catalog_seed)
    return session_mod.Session(obj, box, (0.0, 0.0, 0.0), 1.0, catalog, context=context), obj, box


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=64)
    ap.add_argument("--steps", type=int, default=8, help="placements per job")
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--k", type=int, default=32)
    ap.add_argument("--max-orientations", type=int, default=512)
    ap.add_argument("--weights", default=os.path.join(HERE, "weights", "proposal_rounded256.npz"))
    args = ap.parse_args()
    import torch

    compute, proposal, session_mod = pkg("compute"), pkg("proposal"), pkg("session")
    specs = job_specs(args.jobs, args.seed, args.max_orientations)

    def open_all():
        jobs = []
        for spec in specs:
            ctx = compute.Context(0)
            s, _, _ = open_job(spec, ctx)
            net = proposal.Proposal(context=ctx)
            net.load(args.weights)
            jobs.append((ctx, s, net))
        return jobs

    def close_all(jobs):
        for ctx, s, net in jobs:
            net.close()
            s.close()
            ctx.close()

    t0 = time.perf_counter()
    jobs = open_all()
    open_s = time.perf_counter() - t0
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    together = session_mod.run_jobs([(s, net, args.k, args.steps) for _, s, net in jobs])
    torch.cuda.synchronize()
    concurrent_s = time.perf_counter() - t1
    placed = [len(p) for p, _ in together]
    lengths = [list(s.fft_shape) for _, s, _ in jobs]
    close_all(jobs)

    jobs = open_all()
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    alone = [session_mod.run_jobs([(s, net, args.k, args.steps)])[0] for _, s, net in jobs]
    torch.cuda.synchronize()
    sequential_s = time.perf_counter() - t2
    same = all([(p.orientation_index, p.translation) for p in a[0]] == [(p.orientation_index, p.translation)
                                                                         for p in b[0]]
               for a, b in zip(together, alone))
    close_all(jobs)
    total = sum(placed)
    print(json.dumps({
        "jobs": len(specs), "steps_per_job": args.steps, "k": args.k,
        "windows": [list(s.window) for s in specs], "fft_lengths": lengths,
        "items": [s.item for s in specs], "orientations": [s.orientations for s in specs],
        "placements": total, "fallback_steps": int(sum(fb for _, fb in together)),
        "open_s": round(open_s, 2), "concurrent_s": round(concurrent_s, 3), "sequential_s": round(sequential_s, 3),
        "concurrent_placements_per_s": round(total / concurrent_s, 2),
        "sequential_placements_per_s": round(total / sequential_s, 2),
        "same_placements_concurrent_and_alone": same,
    }))


if __name__ == "__main__":
    main()
