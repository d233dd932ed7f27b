"""Test configuration: the `gpu` marker, seeded RNG, and CUDA availability gating.

Tests marked `gpu` run the CUDA kernels through the C-ABI and need a B200; everything else
(oracle vs golden fixtures, host-side argument logic, C-ABI symbol table, multi-rank logic on
gloo) runs on CPU.
"""

import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA kernels")


def pytest_collection_modifyitems(config, items):
    import torch

    if torch.cuda.is_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture
def rng():
    return np.random.default_rng(1234)
