"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU."""
from __future__ import annotations

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: full-size workloads")


@pytest.fixture(scope="session")
def oracle():
    """The CPU oracle (built from oracle/Makefile; needs the HPMC tree only to build)."""
    from oracle import oracle as O

    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libhpmc_oracle.so")):
        O.build()
    return O


@pytest.fixture(scope="session")
def hpmc():
    import hpmc_b200

    hpmc_b200.lib()  # raises if the CUDA library is missing
    return hpmc_b200
