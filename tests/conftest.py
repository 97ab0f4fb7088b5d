import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def titan():
    """The package (its directory name is not an identifier)."""
    return importlib.import_module("titan_c-_b200")


@pytest.fixture(scope="session")
def built_lib(titan):
    from importlib import import_module

    build = import_module("titan_c-_b200.build")
    build.build()
    return titan.native.lib()


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle_lib as ol

    ol.build_oracle()
    return ol
