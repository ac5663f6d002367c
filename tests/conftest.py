import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")


def package(name=""):
    return importlib.import_module("cpp-max-packer_b200" + ("." + name if name else ""))


@pytest.fixture(scope="session")
def spk():
    return package()


@pytest.fixture(scope="session")
def oracle_c():
    from oracle.bindings import C

    return C()


@pytest.fixture(scope="session")
def oracle_ref():
    from oracle.bindings import REF_SO, Ref

    if not os.path.exists(REF_SO):
        pytest.skip("reference oracle library not built (oracle/ref/Makefile needs the reference sources)")
    return Ref()


@pytest.fixture(scope="session")
def gpu_ctx():
    compute = package("compute")
    ctx = compute.Context(0)
    yield ctx
    ctx.close()
