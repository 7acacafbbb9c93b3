import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

REFERENCE = "/root/reference"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the library and the oracle when their .so files are missing."""
    from dcu_b200 import build as B
    import oracle

    if not os.path.exists(B.LIBNAME) or not os.path.exists(B.CLINAME):
        B.build()
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        oracle.build(REFERENCE if os.path.isdir(REFERENCE) else None)
    yield


@pytest.fixture(scope="session")
def ctx():
    from dcu_b200.api import Context

    c = Context(0)
    yield c
    c.close()


def reference_file(rel):
    p = os.path.join(REFERENCE, rel)
    if not os.path.exists(p):
        pytest.skip(f"reference tree not present ({rel})")
    return p
