"""Shared test setup: the ``gpu`` marker, the golden fixtures and the oracle."""

from __future__ import annotations

import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line(
        "markers",
        "fake_pointers: passes made-up device addresses to the C ABI to check that validation refuses "
        "the call; run with no CUDA device visible, so that a missed check fails on the host",
    )


def _device_visible() -> bool:
    import torch

    return torch.cuda.is_available()


def pytest_pyfunc_call(pyfuncitem):
    """Tests marked ``fake_pointers`` hand addresses such as 16 to the C ABI
    and expect a validation error before any launch.  On a machine with a GPU
    a regression in that validation would launch a kernel on them, so there
    the test runs in a child process that sees no CUDA device
    (``CUDA_VISIBLE_DEVICES=""``): a missed check then fails with a CUDA
    error on the host instead of a memory fault on the device."""
    if pyfuncitem.get_closest_marker("fake_pointers") is None or not _device_visible():
        return None
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-p", "no:cacheprovider", pyfuncitem.nodeid],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, f"{pyfuncitem.nodeid} with no device visible:\n{r.stdout[-4000:]}\n{r.stderr[-2000:]}"
    return True


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
