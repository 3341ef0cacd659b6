import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))
sys.path.insert(0, str(ROOT / "tests" / "golden"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built_library():
    """Make sure libtcs.so and the oracle are built (no-op when up to date)."""
    from threadcoarsenedstencilgenerator_b200.build import build
    from oracle.build import build_oracle

    if os.environ.get("TCS_SKIP_BUILD") != "1":
        build()
    build_oracle()


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
