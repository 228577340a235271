import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built sm_100a library")


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def native():
    """The CUDA library; on a GPU run a missing library is an error, never a skip."""
    from outbreaklab_b200 import build, _native
    build.build()
    return _native


@pytest.fixture(autouse=True)
def _parity_label(request):
    """Labels the parity records (tests/_parity.py) with the running test."""
    try:
        import _parity
    except ImportError:
        yield
        return
    _parity.CURRENT[0] = request.node.nodeid
    yield


def pytest_sessionfinish(session, exitstatus):
    """With OB_PARITY_REPORT=<file>, appends every per-field parity error of the session to it as JSON lines."""
    path = os.environ.get("OB_PARITY_REPORT")
    if not path:
        return
    try:
        import _parity
    except ImportError:
        return
    import json
    with open(path, "a") as f:
        for r in _parity.RECORDS:
            f.write(json.dumps(r) + "\n")
