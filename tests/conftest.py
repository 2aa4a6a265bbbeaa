"""Shared test set-up: the gpu marker and import paths.

Tests marked ``gpu`` need a B200 and the built CUDA library; everything else
runs on CPU (the oracle, the host-side model, the C-ABI symbol table, the
ctypes mirror and the gloo replica tests).
"""

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PACKAGE = os.path.join(ROOT, "spectral-kernel-benchmarks_b200")
for path in (ROOT, PACKAGE):
    if path not in sys.path:
        sys.path.insert(0, path)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device and the built libskb_cuda.so")


@pytest.fixture(scope="session")
def golden_vectors():
    import numpy as np

    return np.load(os.path.join(GOLDEN, "reference_vectors.npz"))


@pytest.fixture(scope="session")
def known_answers():
    import json

    with open(os.path.join(GOLDEN, "known_answers.json")) as fh:
        return json.load(fh)
