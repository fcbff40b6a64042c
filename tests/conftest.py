import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Bring the in-tree CUDA library and the CPU oracle up to date (no-op when fresh)."""
    from lbm3_b200 import build as product_build
    import oracle

    if os.environ.get("LBM3_SKIP_BUILD") != "1":
        product_build.build()
        oracle.build()
    yield
