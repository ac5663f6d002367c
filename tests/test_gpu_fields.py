"""GPU conservative fields and the greedy loop against the reference's own
outputs (golden vectors made by tests/golden/make_golden.py)."""

import os

import numpy as np
import pytest

from conftest import ROOT, package

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(ROOT, "tests", "golden", "fields.npz"))
GREEDY = np.load(os.path.join(ROOT, "tests", "golden", "greedy.npz"))
CASES = ["cuboid", "cuboid_offset", "blob", "blob_fine"]


def _mesh(name, role="object"):
    return package("assets").accept_stl(GOLD[f"{name}/stl"].tobytes(), role=role)


@pytest.mark.parametrize("name", CASES)
def test_object_kernels_bit_exact(gpu_ctx, name):
    geometry = package("geometry")
    mesh = _mesh(name)
    origin, pitch = GOLD[f"{name}/origin"], float(GOLD[f"{name}/pitch"])
    for i, q in enumerate(GOLD[f"{name}/quaternions"]):
        f = geometry.voxelize_object(mesh, origin, pitch, q, context=gpu_ctx)
        assert list(f.first) == list(GOLD[f"{name}/kernel{i}/first"])
        assert list(f.shape) == list(GOLD[f"{name}/kernel{i}/shape"])
        assert np.array_equal(f.cells, GOLD[f"{name}/kernel{i}/cells"]), (name, i)


@pytest.mark.parametrize("name", CASES)
def test_placed_fields_bit_exact(gpu_ctx, name):
    geometry = package("geometry")
    mesh = _mesh(name)
    origin, pitch = GOLD[f"{name}/origin"], float(GOLD[f"{name}/pitch"])
    window = GOLD[f"{name}/placed_window"]
    for i in range(3):
        for clearance in (0.0, 0.8):
            key = f"{name}/placed{i}_{clearance}"
            f = geometry.voxelize_placed(mesh, origin, pitch, window[:3], window[3:], GOLD[key + "/translation"],
                                         GOLD[key + "/q"], clearance, context=gpu_ctx)
            assert np.array_equal(f.cells, GOLD[key]), key


@pytest.mark.parametrize("name", ["box64", "box_odd"])
@pytest.mark.parametrize("clearance", [0.0, 0.9])
def test_box_container_bit_exact(gpu_ctx, name, clearance):
    geometry = package("geometry")
    key = f"container/{name}_{clearance}"
    m = GOLD[key + "/meta"]
    f = geometry.voxelize_container(m[0:3], m[3:6], float(m[6]), m[7:10].astype(np.int64), m[10:13].astype(np.int64),
                                    clearance, context=gpu_ctx)
    assert np.array_equal(f.cells, GOLD[key])


@pytest.mark.parametrize("clearance", [0.0, 1.1])
def test_mesh_container_bit_exact(gpu_ctx, clearance):
    geometry = package("geometry")
    key = f"container/rounded_{clearance}"
    m = GOLD[key + "/meta"]
    f = geometry.voxelize_container(_mesh("container/rounded", "container"), m[0:3], float(m[3]),
                                    m[4:7].astype(np.int64), m[7:10].astype(np.int64), clearance, context=gpu_ctx)
    assert np.array_equal(f.cells, GOLD[key])


@pytest.mark.parametrize("case", [0, 1])
def test_greedy_sequence_matches_reference(gpu_ctx, case):
    assets, session_mod = package("assets"), package("session")
    mesh = assets.accept_stl(GREEDY[f"case{case}/stl"].tobytes())
    s = session_mod.Session(mesh, GREEDY[f"case{case}/box"], (0.0, 0.0, 0.0), 1.0, GREEDY[f"case{case}/catalog"],
                            context=gpu_ctx)
    want_o = GREEDY[f"case{case}/orientations"]
    got = s.greedy(len(want_o))
    assert len(got) == len(want_o)
    for p, o, t, score in zip(got, want_o, GREEDY[f"case{case}/translations"], GREEDY[f"case{case}/scores"]):
        assert p.orientation_index == int(o) and list(p.translation) == list(t)
        assert abs(p.score - score) < 1e-12
    s.close()
