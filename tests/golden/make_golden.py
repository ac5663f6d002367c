"""Regenerates tests/golden/*.npz from the reference's own C++.

Runs the reference hot-path sources compiled here (oracle/_ref/libspk_ref.so,
built from the reference checkout by oracle/ref/Makefile) on seeded synthetic
inputs and stores its outputs as golden vectors for the GPU tests:

    python tests/golden/make_golden.py

fields.npz  - voxelize_object / voxelize_container / voxelize_placed cells and
              windows, oriented bounds, cube catalog (bit-exact references)
greedy.npz  - placement sequences of the reference's page/validate loop for
              configurations without exact score ties
"""

import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.bindings import Ref, ref_voxelize_container  # noqa: E402

syn = importlib.import_module("cpp-max-packer_b200.synthetic")


def random_quaternions(rng, n):
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1)[:, None]
    return q


def object_cases(ref):
    """(name, stl, origin, pitch, quaternions)."""
    rng = np.random.default_rng(20)
    cube = ref.catalog(1)
    return [
        ("cuboid", syn.cuboid_stl(), (0.0, 0.0, 0.0), 1.0, cube),
        ("cuboid_offset", syn.cuboid_stl((7.5, 3.25, 4.0)), (0.13, -0.27, 0.05), 0.5, cube[::5]),
        ("blob", syn.blob_stl(3, level=2, radius_range=(3.0, 4.0)), (0.0, 0.0, 0.0), 0.5,
         ref.catalog(4, random_quaternions(rng, 6))),
        ("blob_fine", syn.blob_stl(4, level=3, radius_range=(4.0, 6.0)), (0.31, 0.17, -0.4), 0.7,
         ref.catalog(4, random_quaternions(rng, 4))),
    ]


def main():
    ref = Ref()
    out = {}
    out["cube_catalog"] = ref.catalog(1)
    for name, stl, origin, pitch, quats in object_cases(ref):
        asset = ref.asset(stl)
        v, t, b = asset.mesh()
        out[f"{name}/stl"] = np.frombuffer(stl, np.uint8)
        out[f"{name}/vertices"], out[f"{name}/triangles"] = v, t
        out[f"{name}/origin"], out[f"{name}/pitch"] = np.array(origin), np.array(pitch)
        out[f"{name}/quaternions"] = quats
        for i, q in enumerate(quats):
            first, shape, cells = asset.voxelize_object(origin, pitch, q)
            out[f"{name}/kernel{i}/first"], out[f"{name}/kernel{i}/shape"] = first, shape
            out[f"{name}/kernel{i}/cells"] = cells
            out[f"{name}/bounds{i}"] = asset.oriented_bounds(q)
        # placed copies over a fixed window, with and without pair clearance
        rng = np.random.default_rng(len(name))
        wfirst, wshape = np.array([-3, -4, -2]), np.array([30, 26, 22], np.uint32)
        out[f"{name}/placed_window"] = np.concatenate([wfirst, wshape]).astype(np.int64)
        for i in range(3):
            q = quats[i % len(quats)]
            tr = origin + pitch * rng.integers(2, 12, size=3) + rng.uniform(-0.3, 0.3, size=3) * (i == 2)
            for clearance in (0.0, 0.8):
                cells = asset.voxelize_placed(origin, pitch, wfirst, wshape, tr, q, clearance)
                key = f"{name}/placed{i}_{clearance}"
                out[key], out[key + "/translation"], out[key + "/q"] = cells, np.array(tr), q
    # containers
    for name, container, origin, pitch, first, shape in [
        ("box64", (64.0, 64.0, 64.0), (0.0, 0.0, 0.0), 1.0, (-1, -1, -1), (66, 66, 66)),
        ("box_odd", (20.3, 17.9, 12.25), (0.1, -0.2, 0.05), 0.45, (-2, -1, -2), (49, 43, 31)),
    ]:
        for clearance in (0.0, 0.9):
            cells = ref_voxelize_container(ref, container, origin, pitch, first, shape, clearance)
            out[f"container/{name}_{clearance}"] = cells
            out[f"container/{name}_{clearance}/meta"] = np.array([*container, *origin, pitch, *first, *shape])
    stl = syn.rounded_box_stl((12.0, 10.0, 9.0), exponent=4.0, level=3)
    casset = ref.asset(stl, container=True)
    v, t, b = casset.mesh()
    out["container/rounded/stl"] = np.frombuffer(stl, np.uint8)
    out["container/rounded/vertices"], out["container/rounded/triangles"] = v, t
    for clearance in (0.0, 1.1):
        first, shape = (-1, -1, -1), (27, 23, 21)
        cells = ref_voxelize_container(ref, casset, (0.0, 0.0, 0.0), 1.0, first, shape, clearance)
        out[f"container/rounded_{clearance}"] = cells
        out[f"container/rounded_{clearance}/meta"] = np.array([0, 0, 0, 1.0, *first, *shape])
    np.savez_compressed(os.path.join(HERE, "fields.npz"), **out)

    # greedy sequences (no exact ties: asymmetric blob, random catalog)
    greedy = {}
    rng = np.random.default_rng(77)
    for k, (seed, box, n_orient, steps) in enumerate([(5, (22.0, 18.0, 16.0), 4, 6), (6, (18.0, 16.0, 20.0), 6, 5)]):
        stl = syn.blob_stl(seed, level=2, radius_range=(3.0, 4.0))
        asset = ref.asset(stl)
        catalog = ref.catalog(4, random_quaternions(rng, n_orient))
        session = ref.session(asset, box, 0.0, 0.0, (0.0, 0.0, 0.0), 1.0, catalog)
        ori, t, scores, rejected, seconds = session.greedy(steps)
        greedy[f"case{k}/stl"] = np.frombuffer(stl, np.uint8)
        greedy[f"case{k}/box"] = np.array(box)
        greedy[f"case{k}/catalog"] = catalog
        greedy[f"case{k}/orientations"], greedy[f"case{k}/translations"] = ori, t
        greedy[f"case{k}/scores"] = scores
        print(f"greedy case{k}: {len(ori)} placements in {seconds:.1f}s")
    np.savez_compressed(os.path.join(HERE, "greedy.npz"), **greedy)


if __name__ == "__main__":
    main()
