import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def built():
    """Builds the native libraries in-tree when they are missing."""
    from nectarrender_b200 import LIB_PATH
    from nectarrender_b200.build import MODULE
    import oracle
    if not LIB_PATH.exists() or not MODULE.exists():
        from nectarrender_b200 import build
        build.build_all()
    if not oracle.ORACLE_SO.exists():
        oracle.build(reference_root="")
    yield
