import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)



def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the library and the oracle when their .so files are missing."""
    from dcu_b200 import build as B
    import oracle

    if not all(os.path.exists(p) for p in (B.LIBNAME, B.CLINAME, B.CLI_SINGLE)):
        B.build()
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        oracle.build(oracle.REFERENCE if oracle.reference_present() else None)
    yield


@pytest.fixture(scope="session")
def ctx():
    from dcu_b200.api import Context

    c = Context(0)
    yield c
    c.close()


def reference_file(rel):
    """A reference fixture ("matrices/<name>"): the copy staged with the built
    oracle files, else the reference tree; skip when neither has it."""
    import oracle

    p = oracle.fixture_path(os.path.basename(rel))
    if p is None:
        pytest.skip(f"reference fixture not present ({rel})")
    return p
