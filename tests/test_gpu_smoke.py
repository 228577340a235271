"""The entry point's smoke run (two steps of a small case on cuda:0 against the FP32 and FP64 oracles)."""
import os
import sys

import pytest

pytestmark = pytest.mark.gpu


def test_smoke(native):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import __graft_entry__ as entry
    entry.smoke()
