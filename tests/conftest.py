"""Shared test setup: the ``gpu`` marker, the golden fixtures and the oracle."""

from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def pytest_collection_modifyitems(config, items):
    import torch

    if torch.cuda.is_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def golden():
    return np.load(os.path.join(ROOT, "tests", "golden", "golden.npz"))


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.lib()
    return O


def rel_l2(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.linalg.norm(b.ravel().astype(np.complex128))
    num = np.linalg.norm((a.astype(np.complex128) - b.astype(np.complex128)).ravel())
    return float(num / den) if den > 0 else float(num)
