"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs
on CPU.  The oracle (reference library + C restatement) is test
infrastructure and is loaded only here and in the test modules."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "stars-h_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU")


@pytest.fixture(scope="session")
def ref():
    import oracle
    if not os.path.exists(oracle.REF_SO):
        oracle.build()
    return oracle.Ref()


@pytest.fixture(scope="session")
def orc():
    import oracle
    if not os.path.exists(oracle.ORACLE_SO):
        oracle.build()
    return oracle.Oracle()


@pytest.fixture(scope="session")
def lib():
    import starsh_b200
    if not os.path.exists(starsh_b200.LIB_PATH):
        import build as b200_build
        b200_build.build()
    return starsh_b200.load()
