"""Shared fixtures.  Tests that need a B200 carry @pytest.mark.gpu; the rest
run on a CPU-only machine (oracle pins, ABI exports, translator code
generation compiled with NVRTC)."""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200)")


@pytest.fixture(scope="session")
def chai_dev():
    """One back-end context for the whole GPU session (chai::init)."""
    import chai_b200.api as ch
    os.environ.setdefault("CHAI_JIT_CACHE", str(ROOT / "chai_b200" / "_jitcache"))
    Path(os.environ["CHAI_JIT_CACHE"]).mkdir(exist_ok=True)
    dev = ch.init()
    yield dev
    ch.shutdown()
