import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


@pytest.fixture(scope="session")
def built():
    """Builds (if stale) the library, the generator and the oracle."""
    from ferrousalign_b200 import build as B
    from oracle import build_oracle
    B.build_all()
    build_oracle.build()
    return True


@pytest.fixture(scope="session")
def ctx(built):
    import ferrousalign_b200 as fa
    c = fa.Context(0)
    yield c
    c.close()
