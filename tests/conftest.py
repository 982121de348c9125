import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")
    config.addinivalue_line("markers", "slow: longer CPU-side checks")


@pytest.fixture(scope="session", autouse=True)
def built():
    """Builds libphx.so and the oracle in-tree if missing (no-op when up to date)."""
    from phosphor_b200.build import build_library, build_oracle
    if not os.environ.get("PHX_SKIP_BUILD"):
        build_library()
        build_oracle()
    yield
