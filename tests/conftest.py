import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (run with -m gpu)")
    config.addinivalue_line("markers", "slow: long CPU-oracle runs")


@pytest.fixture(scope="session")
def oracle():
    from oracle_lib import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle_lib import Reference
    if not Reference.available():
        pytest.skip("reference library oracle/_ref/liblcurve_ref.so not built here")
    return Reference()


def _engine(precision):
    from lcurve_re_b200.engine import Engine
    return Engine(precision=precision)


@pytest.fixture(scope="session")
def engine_mixed():
    e = _engine("mixed")
    yield e
    e.close()


@pytest.fixture(scope="session")
def engine_fp64():
    e = _engine("fp64")
    yield e
    e.close()
