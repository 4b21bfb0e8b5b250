import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
for _p in (ROOT, ROOT / "tests"):
    if str(_p) not in sys.path:
        sys.path.insert(0, str(_p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle
    oracle.build()
    return oracle.load()


@pytest.fixture(scope="session")
def gpu_lib():
    """Loads the CUDA library; fails loudly if it was not built (no CPU fallback)."""
    from naivetrace_b200 import abi, build
    build.build()
    return abi.load_library()
