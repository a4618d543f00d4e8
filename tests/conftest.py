import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT / "openstc-mixinglayer_b200" / "python", ROOT / "oracle", ROOT):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def built():
    """Builds the CUDA library (if sources changed) and the CPU oracle."""
    import oracle
    sys.path.insert(0, str(ROOT / "openstc-mixinglayer_b200"))
    import build as libbuild
    libbuild.build()
    oracle.build()
    return True
