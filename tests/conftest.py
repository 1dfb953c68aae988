import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on a B200)")


@pytest.fixture(scope="session")
def built_oracle():
    """Builds oracle/libpdx_port.so (and oracle/_ref when the reference sources exist)."""
    from __graft_entry__ import build_oracles
    build_oracles()
    return True
