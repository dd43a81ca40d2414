import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    """The CPU oracle is test infrastructure; build it if this checkout lacks it."""
    so = os.path.join(ROOT, "oracle", "libsnn_oracle.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), os.path.join(ROOT, "oracle", "libsnn_oracle.so")],
                       check=True)
    yield


def golden_cases(prefix=""):
    gdir = os.path.join(ROOT, "tests", "golden")
    names = sorted(f[:-4] for f in os.listdir(gdir) if f.endswith(".npz"))
    return [n for n in names if n.startswith(prefix)] if prefix else names
