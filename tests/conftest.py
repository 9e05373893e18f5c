import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "reference: needs the compiled reference build in oracle/_ref")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    if not O.LIB_PATH.exists():
        pytest.fail(f"oracle library not built: {O.LIB_PATH} (make -C oracle)")
    return O
