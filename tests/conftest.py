import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "mpfs250t-sar-ifp_b200"
for p in (str(ROOT), str(PKG)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built sm_100a library")
    config.addinivalue_line("markers", "reference: needs the read-only reference checkout (CPU only)")
    config.addinivalue_line("markers", "slow: long-running case")


def reference_available() -> bool:
    from oracle import refshim
    return refshim.available()


@pytest.fixture(scope="session")
def ref_modules():
    from oracle import refshim
    if not refshim.available():
        pytest.skip("reference checkout not present")
    return refshim.modules()


@pytest.fixture(scope="session")
def golden_dir():
    return ROOT / "tests" / "golden"
