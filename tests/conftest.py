"""Test configuration.

Markers: ``gpu`` tests need a CUDA device and call the product through the C
ABI (libproteus_gpu.so); everything else runs on CPU.  The oracle libraries
(oracle/liboracle.so, oracle/_ref/*.so) are the checkers; see oracle/.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libproteus_gpu.so")


@pytest.fixture(scope="session")
def golden2():
    return dict(np.load(os.path.join(GOLDEN, "ref_2d_k16.npz")))


@pytest.fixture(scope="session")
def golden3():
    return dict(np.load(os.path.join(GOLDEN, "ref_3d.npz")))


def ref_available(dim, k):
    import refbuild
    return refbuild.available(dim, k)
