"""Throughput of the validator broad phase (spk_broad_phase) on a layout of
the size of a full fill.

    python cpp-max-packer_b200/broad_phase_bench.py [--copies 3580] [--repeats 20]

The layout stands in for a full fill of the 256^3 rounded container: the
bench item (8,192-triangle blob) at seeded SO(3) rotations, translated
uniformly over a 256 mm cube, with the posed bounds computed by
spk_posed_bounds.  Every pair is visited (a full geometry::validate; no copy
proven).  Printed: pairs per second for the device call end to end (host
bounds in, unresolved pairs out) and the number of unresolved pairs.
bench.py reports the same figure beside the oracle's plain-C loop.
"""

from __future__ import annotations

import argparse
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


def poses(copies: int, seed: int = 3):
    """(item mesh, its STL bytes, translations (copies, 3), quaternions
    (copies, 4)): seeded poses of the bench item over a 256 mm cube."""
    workloads = pkg("workloads")
    spec = workloads.SPECS["rounded256_blob_hopf512"]()
    obj = pkg("assets").accept_stl(spec.object_stl)
    rng = np.random.default_rng(seed)
    q = rng.normal(size=(copies, 4))
    q /= np.linalg.norm(q, axis=1)[:, None]
    q[q[:, 3] < 0] *= -1
    t = rng.uniform(0.0, 256.0, size=(copies, 3))
    return obj, spec.object_stl, t, q


def layout(copies: int, seed: int = 3):
    """(posed bounds min, max, finite) of `copies` seeded poses of the bench item."""
    obj, _, t, q = poses(copies, seed)
    return pkg("geometry").posed_bounds(obj, t, q)


def time_device(lo, hi, fin, clearance: float, repeats: int, context):
    """(seconds per spk_broad_phase call, end to end, after one warm-up call; the pairs)."""
    geometry = pkg("geometry")
    got = geometry.broad_phase(lo, hi, fin, clearance, context=context)
    t0 = time.perf_counter()
    for _ in range(repeats):
        got = geometry.broad_phase(lo, hi, fin, clearance, context=context)
    return (time.perf_counter() - t0) / repeats, got


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--copies", type=int, default=3580)
    ap.add_argument("--repeats", type=int, default=20)
    ap.add_argument("--clearance", type=float, default=0.0)
    args = ap.parse_args()
    compute = pkg("compute")
    lo, hi, fin = layout(args.copies)
    n = args.copies
    pairs = n * (n - 1) // 2
    ctx = compute.Context(0)
    seconds, got = time_device(lo, hi, fin, args.clearance, args.repeats, ctx)
    ctx.close()
    print(json.dumps({"copies": n, "pairs": pairs, "unresolved": int(len(got)),
                      "device_call_ms": round(seconds * 1e3, 3), "device_pairs_per_s": round(pairs / seconds, 1)}))


if __name__ == "__main__":
    main()
