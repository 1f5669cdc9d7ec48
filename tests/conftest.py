import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    """Build the CPU oracles if they are missing (the C restatement always,
    the reference library where the reference sources exist)."""
    import subprocess
    out = os.path.join(ROOT, "oracle", "_ref")
    targets = []
    if not os.path.exists(os.path.join(out, "libnnpport.so")):
        targets.append("port")
    ref = os.environ.get("N2P2_REFERENCE") or os.path.join(os.path.dirname(ROOT), "reference")
    if not os.path.exists(os.path.join(out, "libnnpref.so")) and os.path.isdir(os.path.join(ref, "src", "libnnp")):
        targets.append("ref")
    if targets:
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "-j8", "N2P2_REFERENCE=" + ref, *targets],
                       check=False, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    yield
