"""Shared pytest configuration.

Markers:
  gpu -- needs a CUDA device (B200, sm_100a); run with `-m gpu`.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "nemolite2d-cuda_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a)")


GOLDEN = os.path.join(ROOT, "tests", "golden")
GOLDEN_CASES = ["g10x10_ref128phys", "g16x9_ref128phys", "g9x14_defaultphys",
                "g32x32_ref128phys", "g128x128_cfg0"]


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.build()
    return oracle
