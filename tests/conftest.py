import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); calls the CUDA path through the C ABI")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Build the oracle and the CUDA library in-tree once per session (no-ops when current)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    if not os.path.exists(os.path.join(ROOT, "repulsor_b200", "librepulsor_b200.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "repulsor_b200")], check=True)
    yield
