import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_lib():
    """The CPU restatement (the parity checker), built from oracle/ on first use."""
    from tests.oracle_lib import oracle_library

    return oracle_library()


@pytest.fixture(scope="session")
def cuda_lib():
    from ironav_b200 import build
    from ironav_b200.inter import cuda_library

    build.build_cuda()
    return cuda_library()
