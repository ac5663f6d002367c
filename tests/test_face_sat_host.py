"""The raster's per-face separating-axis data (face_sat / face_sat_disjoint,
csrc/interval.cuh) against the per-cell test it replaces
(triangle_box_disjoint, the restatement of validation_kernel.cpp's
triangle-box SAT): tests/native/face_sat_check.cu compares the two on 2.4 M
seeded triangle/cell pairs on the host, with degenerate triangles, widened
vertex intervals and overflowing magnitudes."""

import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def test_face_sat_matches_the_per_cell_test(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc is not available")
    exe = str(tmp_path / "face_sat_check")
    subprocess.run([nvcc, "-O2", "-std=c++17", "--expt-relaxed-constexpr", "-gencode",
                    "arch=compute_100a,code=sm_100a", "-o", exe, os.path.join(HERE, "native", "face_sat_check.cu")],
                   check=True, capture_output=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    cases, disjoint = int(out.stdout.split()[0]), int(out.stdout.split()[2])
    assert cases > 1_000_000 and 0.2 * cases < disjoint < 0.8 * cases
