import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


_SYSTEMS = {}


def get_system(name):
    from west_b200.system import build_system
    if name not in _SYSTEMS:
        _SYSTEMS[name] = build_system(name)
    return _SYSTEMS[name]


@pytest.fixture(scope="session")
def tiny():
    return get_system("tiny")


@pytest.fixture(scope="session")
def small():
    return get_system("small")
