import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer CPU oracle runs")


@pytest.fixture(scope="session")
def ref_harness():
    """The unmodified reference compiled under oracle/_ref (built by build())."""
    import refio

    if not os.path.exists(refio.REF_HARNESS):
        import importlib

        ref_src = importlib.import_module("__graft_entry__").reference_src()
        if os.path.isdir(ref_src):
            import subprocess

            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), f"REF={ref_src}", "ref"], check=True,
                           stdout=subprocess.DEVNULL)
        else:
            pytest.skip("reference build oracle/_ref/ref_harness not present")
    return refio.REF_HARNESS
