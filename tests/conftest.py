import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

REF_DIR = "/root/reference"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run with -m gpu)")


@pytest.fixture(scope="session")
def oracle3():
    from oracle.pyoracle import Oracle
    return Oracle(3)


@pytest.fixture(scope="session")
def oracle2():
    from oracle.pyoracle import Oracle
    return Oracle(2)


def reference_lib(kind):
    """The reference compiled from source (oracle/_ref), or skip when absent."""
    from oracle.pyoracle import HERE, Reference
    path = os.path.join(HERE, "_ref", Reference.LIBS[kind][0])
    if not os.path.exists(path) and not os.path.isdir(REF_DIR):
        pytest.skip("reference build oracle/_ref not available")
    return Reference(kind)
