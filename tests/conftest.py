import os
import sys
from pathlib import Path

# hardware work queues for the serving runtime's streams (read when the CUDA context is created)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds libgq.so and the oracle once per session (no-op when up to date)."""
    from gquery_b200 import build_lib
    import oracle
    if not (os.environ.get("GQ_SKIP_BUILD") and build_lib.LIB.exists()):
        build_lib.build()
    oracle.build()
    yield
