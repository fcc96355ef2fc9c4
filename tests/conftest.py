import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)



def _reference_dir():
    """Where the reference sources are: the MPS_REFERENCE_DIR environment
    variable, else the directory oracle/_ref was compiled from (recorded by
    oracle/Makefile in oracle/_ref/SOURCES); None when neither exists on this
    machine (tests that read reference files then skip)."""
    d = os.environ.get("MPS_REFERENCE_DIR")
    if not d:
        stamp = os.path.join(ROOT, "oracle", "_ref", "SOURCES")
        if os.path.exists(stamp):
            for line in open(stamp):
                if line.startswith("# "):
                    d = line.split(maxsplit=2)[2].strip()
                    break
    return d if d and os.path.isdir(d) else None


REF_DIR = _reference_dir()


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
    if not os.path.exists(path):
        pytest.skip("reference build oracle/_ref not available (build it with make -C oracle, "
                    "MPS_REFERENCE_DIR naming the reference checkout)")
    return Reference(kind)
