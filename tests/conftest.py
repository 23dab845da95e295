import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def ref():
    """The reference's own CPU code (oracle/_ref), the checker for parity."""
    from oracle import ref as r
    if not r.available():
        pytest.fail("oracle/_ref/libfrost_ref.so is not built (make -C oracle ref)")
    return r
