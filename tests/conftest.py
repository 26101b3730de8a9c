import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the parity tests")


@pytest.fixture(scope="session")
def gsb():
    import gsb200

    return gsb200


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle_py

    return oracle_py
