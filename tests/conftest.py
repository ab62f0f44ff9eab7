"""Shared fixtures: paths, the oracle (checker) and the product library."""
import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "gadget-ng_b200")
for p in (REPO, PKG, os.path.join(REPO, "oracle"), os.path.dirname(os.path.abspath(__file__))):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: CPU test that takes more than a few seconds")


def oracle():
    """The CPU restatement (test infrastructure; never used by the product)."""
    import oracle as _o
    return _o
