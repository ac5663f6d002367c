"""The maintainer-side adapter (cpp-max-packer_b200/integration/) compiled
against the reference's own correlation headers and checked against the
reference's correlate_binary_cpu / correlate_proximity_cpu from the
reference build.

On a host without a GPU this covers what the adapter decides itself:
- the stop token and deadline, through a replaced clock;
- the extent, translation-range and cell-count checks, in the reference's
  order and with its codes;
- failing closed with CORRELATION_ALLOCATION where the device would be
  needed.
With a device the same binary also compares the values.  It needs the
reference checkout, for its headers, and is skipped without it.
"""

import os
import subprocess

import pytest

from conftest import ROOT
from oracle.bindings import REF_SO, REFERENCE_ROOT

HERE = os.path.join(ROOT, "tests", "adapter")
LIB = os.path.join(ROOT, "cpp-max-packer_b200", "libspk_b200.so")


@pytest.mark.timeout(300)
def test_adapter_matches_reference_contract():
    headers = os.path.join(REFERENCE_ROOT, "engine", "pack_compute", "include")
    if not os.path.isdir(headers) or not os.path.exists(REF_SO) or not os.path.exists(LIB):
        pytest.skip("needs the reference headers, the reference build and libspk_b200.so")
    subprocess.run(["make", "-s", "-C", HERE, f"REF={REFERENCE_ROOT}"], check=True)
    run = subprocess.run([os.path.join(HERE, "_build", "adapter_check")], capture_output=True, text=True,
                         timeout=120)
    assert run.returncode == 0 and run.stdout.strip().endswith("PASS"), run.stdout + run.stderr
    lines = run.stdout.splitlines()
    for case in ("binary", "proximity", "stopped", "deadline", "invalid_field", "zero_extent", "index_overflow",
                 "invalid_kernel", "mask"):
        assert any(line.startswith(f"ok {case} ") for line in lines), run.stdout
