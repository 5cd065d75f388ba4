import os
import sys

import pytest

REPO = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
for p in (os.path.join(REPO, "ho-cxx_b200"), os.path.join(REPO, "oracle"), REPO):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(REPO, "tests", "golden")


def reference_root() -> str:
    """Root of the reference's sources, read by the tests that compare with them:
    $HO2D_REFERENCE, else the reference checkout of the build machine (absent elsewhere)."""
    return os.environ.get("HO2D_REFERENCE") or "/root/reference"


GOLDEN_CASES = sorted(d for d in os.listdir(GOLDEN) if os.path.isfile(os.path.join(GOLDEN, d, "ref.npz")))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
