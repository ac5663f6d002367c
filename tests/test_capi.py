"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: CPU only)."""

import glob
import os
import re

from conftest import ROOT, package


def declared_symbols():
    names = set()
    for header in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(header).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(spk_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    lib = package("_lib").lib()
    names = declared_symbols()
    assert "spk_correlate_binary" in names
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_status_codes_map_to_reference_strings():
    lib = package("_lib")
    assert lib.status_code(0) == "OK"
    assert lib.status_code(9) == "CORRELATION_NUMERIC"
    assert lib.status_code(7) == "CORRELATION_PADDED_CELL_LIMIT"
    assert lib.status_code(12) == "OPERATION_CANCELLED"
    assert lib.status_code(13) == "DEADLINE_EXCEEDED"


def test_estimate_is_host_only():
    compute = package("compute")
    est = compute.estimate_correlation(compute.CorrelationSpec((66, 66, 66), (12, 16, 22)))
    # The transform length per axis is the smallest 2^a 3^b 5^c >= E + K - 1.
    assert est.padded_shape == (80, 81, 90)
    assert est.padded_cells == 77 * 81 * 87
