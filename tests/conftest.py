import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA library")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    from coupled_cluster_doubles_b200 import build
    from oracle.build import build_oracle
    build.build_host()
    build_oracle()
    yield
