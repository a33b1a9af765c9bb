"""Shared fixtures.  ``-m gpu`` tests need a CUDA device and the built
library; everything else runs on the CPU."""

import importlib
import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

GOLDEN = os.path.join(REPO, "tests", "golden", "reference_vectors.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the sm_100a library")


@pytest.fixture(scope="session")
def h3():
    return importlib.import_module("3dhit_b200")


@pytest.fixture(scope="session")
def orc():
    from oracle import hit3d_oracle
    return hit3d_oracle


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(GOLDEN))


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


# golden cases: tag -> (dims, numpy dtype)
CASES = {
    "c16f": ((16, 16, 16), np.float32),
    "c32f": ((32, 32, 32), np.float32),
    "c16x8x4d": ((16, 8, 4), np.float64),
    "c16d": ((16, 16, 16), np.float64),
    "a16x32x8f": ((16, 32, 8), np.float32),
}
