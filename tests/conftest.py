import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle.oracle import Reference
    if not Reference.available():
        pytest.skip("reference core not built (oracle/_ref absent)")
    return Reference()


@pytest.fixture(scope="session")
def ses():
    import shoeridingerequationsolver_b200 as s
    if s.device_count() < 1:
        pytest.fail("no CUDA device visible to libses_b200.so")
    return s
