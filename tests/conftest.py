import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT / "delayed-pivoting_b200", ROOT / "oracle", ROOT / "tests"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "slow: long-running case")


@pytest.fixture(scope="session")
def built():
    """Builds the oracle (and the reference CPU build when its sources exist)."""
    import oracle

    oracle.build(ref=True)
    return True
