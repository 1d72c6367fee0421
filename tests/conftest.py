import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs libedk kernels)")


@pytest.fixture(scope="session")
def O():
    """The CPU oracle (test infrastructure)."""
    import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def ek():
    """The product package (edkit.jl_b200/ imported as edkit_b200).  Fails if
    libedk.so was built from sources other than the ones in the tree."""
    import importlib.util
    import __graft_entry__ as ge
    mod = ge.load_package()
    spec = importlib.util.spec_from_file_location(
        "edk_build", os.path.join(ROOT, "edkit.jl_b200", "build.py"))
    bld = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bld)
    want = bld.source_hash()
    have = mod.version().rsplit(" ", 1)[-1]
    assert have == want, f"libedk.so is stale (built from {have}, sources are {want})"
    return mod
