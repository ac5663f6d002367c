"""Regenerates tests/golden/sequences.npz: placement sequences of the
reference's own greedy on the benchmark-shaped workloads.

Runs the reference hot-path sources compiled here (oracle/_ref/libspk_ref.so)
through its page/validate loop (spectral.cpp:1460-1591 with try_pose ->
geometry::validate_incremental, restated around the reference's functions in
oracle/ref/ref_api.cpp) on the seeded workloads of the package's
workloads.SPECS, with the catalog canonicalised by the reference's own
make_orientation_catalog.  Each case stores the reference's sequence
(orientation, translation, score), the number of validator rejections and the
SHA-256 of the inputs, so the GPU tests can rebuild the same workload without
the reference:

    python tests/golden/make_sequences.py [case ...]

Cases (each runs in its own process; the file is rewritten as each ends):
  cuboid66   box 64 mm at 1 mm (66^3 window), 10x14x20 mm cuboid, the 24 cube
             rotations, greedy to completion (at most 80 copies)
  blob128    box 63 mm at 0.5 mm (128^3 window), 5,120-triangle blob, the first
             16 of the 96 seeded SO(3) orientations, 12 copies
  rounded256 rounded-box container STL (256^3 window), 8,192-triangle blob,
             the first 4 of the 512 seeded SO(3) orientations, 3 copies
"""

import hashlib
import importlib
import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

CASES = {
    # name: (workload, orientations used, steps)
    "cuboid66": ("box64_cuboid_cube24", 24, 80),
    "blob128": ("box63_blob_hopf96", 16, 12),
    "rounded256": ("rounded256_blob_hopf512", 4, 3),
}


def sha(data: bytes) -> str:
    return hashlib.sha256(data).hexdigest()


def run_case(name):
    from oracle.bindings import Ref

    workloads = importlib.import_module("cpp-max-packer_b200.workloads")
    workload, n_orient, steps = CASES[name]
    spec = workloads.SPECS[workload]()
    ref = Ref()
    obj = ref.asset(spec.object_stl)
    container = tuple(spec.container_box) if spec.container_box is not None else \
        ref.asset(spec.container_stl, container=True)
    catalog = ref.catalog(1) if spec.catalog_kind == "cube" else ref.catalog(4, spec.raw_quaternions())
    catalog = catalog[:n_orient]
    session = ref.session(obj, container, spec.pair_clearance, spec.wall_clearance, spec.origin, spec.pitch, catalog)
    t0 = time.time()
    ori, t, scores, rejected, seconds = session.greedy(steps)
    out = {
        f"{name}/workload": np.array(workload),
        f"{name}/object_sha256": np.array(sha(spec.object_stl)),
        f"{name}/container_sha256": np.array(sha(spec.container_stl)),
        f"{name}/catalog": catalog,
        f"{name}/orientations": ori.astype(np.int64),
        f"{name}/translations": t,
        f"{name}/scores": scores,
        f"{name}/rejected": np.array(rejected),
        f"{name}/steps_requested": np.array(steps),
        f"{name}/seconds": np.array(seconds),
    }
    print(f"{name}: {len(ori)} placements, {rejected} rejected, {time.time() - t0:.1f} s", flush=True)
    return name, out


def main(names):
    path = os.path.join(HERE, "sequences.npz")
    with mp.get_context("spawn").Pool(len(names)) as pool:
        for name, out in pool.imap_unordered(run_case, names):
            merged = dict(np.load(path, allow_pickle=False)) if os.path.exists(path) else {}
            merged = {k: v for k, v in merged.items() if not k.startswith(name + "/")}
            merged.update(out)
            np.savez_compressed(path, **merged)


if __name__ == "__main__":
    main(sys.argv[1:] or list(CASES))
