import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
LAMBDA = os.path.join(GOLDEN, "lambda")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the device path through the C ABI)")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.load()
    return oracle


@pytest.fixture(scope="session")
def native_lib():
    from racon_b200 import build
    build.build()
    import racon_b200
    return racon_b200


def lambda_path(name):
    return os.path.join(LAMBDA, name)
