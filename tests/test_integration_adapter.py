"""The maintainer-side adapter (cpp-max-packer_b200/integration/) compiled
against the reference's own correlation headers and checked against the
reference's correlate_binary_cpu / correlate_proximity_cpu from the
reference build.

On a host without a GPU this covers what the adapter decides itself:
- the metadata limit, then the stop token and deadline (through a replaced
  clock), in the reference's order;
- the extent, translation-range and cell-count checks, in the reference's
  order and with its codes and per-site messages;
- failing closed with CORRELATION_ALLOCATION where the device would be
  needed.
With a device (the gpu-marked test) the same binary also compares the
values, and the failures the library itself reports carry the reference's
message for the site.  Building the check needs the reference checkout, for
its headers; the gpu test runs the binary built here, which travels with the
tree.
"""

import os
import subprocess

import pytest

from conftest import ROOT
from oracle.bindings import REF_SO

HERE = os.path.join(ROOT, "tests", "adapter")
LIB = os.path.join(ROOT, "cpp-max-packer_b200", "libspk_b200.so")
CHECK = os.path.join(HERE, "_build", "adapter_check")
CASES = ("binary", "proximity", "stopped", "deadline", "invalid_field", "zero_extent", "index_overflow",
         "stopped_no_memory", "last_translation", "invalid_environment", "padded_limit", "invalid_kernel", "mask")


def _run_check():
    run = subprocess.run([CHECK], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0 and run.stdout.strip().endswith("PASS"), run.stdout + run.stderr
    lines = run.stdout.splitlines()
    for case in CASES:
        assert any(line.startswith(f"ok {case} ") for line in lines), run.stdout
    return lines


@pytest.mark.timeout(300)
def test_adapter_matches_reference_contract():
    if not os.path.exists(REF_SO) or not os.path.exists(LIB):
        pytest.skip("needs the reference build and libspk_b200.so")
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if not os.path.exists(CHECK):
        pytest.skip("the reference headers are absent, so the adapter check cannot be built here")
    _run_check()


@pytest.mark.gpu
@pytest.mark.timeout(300)
def test_adapter_values_on_device():
    """On the device the adapter's values equal the reference's: binary
    counts exactly, proximity within the reference's 1e-10, and the device
    mask equals the mask rule applied to the reference's counts."""
    if not os.path.exists(CHECK):
        pytest.fail("tests/adapter/_build/adapter_check is missing: build it where the reference headers are")
    lines = _run_check()
    for case in ("binary", "proximity", "mask", "padded_limit", "invalid_environment"):
        line = next(line for line in lines if line.startswith(f"ok {case} "))
        assert "no device" not in line, line
