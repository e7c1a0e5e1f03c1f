import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

MECH = os.path.join(ROOT, "janc_b200", "mechanisms", "9sp-19r-H2-Air.yaml")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session")
def mech_path():
    return MECH


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN
