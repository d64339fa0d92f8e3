"""Shared pytest configuration.

Markers:
  gpu  -- needs a CUDA device and the built extension (run with ``-m gpu``).
  slow -- long CPU cases.
"""

import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")
DEFAULT_SEED = 8966433580120847635


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: requires a CUDA GPU and the built extension")
    config.addinivalue_line("markers", "slow: long-running CPU case")


@pytest.fixture(scope="session")
def golden():
    data = np.load(os.path.join(GOLDEN_DIR, "golden.npz"))
    with open(os.path.join(GOLDEN_DIR, "golden_index.json")) as fh:
        index = json.load(fh)
    return data, index


@pytest.fixture
def rng():
    return np.random.default_rng(DEFAULT_SEED)


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
