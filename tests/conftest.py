"""Shared set-up of the tests.

* ``@pytest.mark.gpu`` marks the tests that need a CUDA device (the parity
  tests of the kernels proper, which call the C-ABI library); the CPU suite
  is ``pytest -m "not gpu"``.
* The repository root is importable (``oracle``, ``waveformx_b200``).
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); calls the kernels through the C-ABI")


def golden(name):
    """A golden fixture (``tests/golden/<name>.npz``) as a dict of arrays."""
    with np.load(GOLDEN / f"{name}.npz") as data:
        return {k: data[k] for k in data.files}


def compare(test, reference):
    """``(max |a - b| / max |b|, mismatch)`` with uniform weights, per the
    reference's shared metric (its ``tests/conftest.py:65-75``)."""
    test = np.asarray(test)
    reference = np.asarray(reference)
    assert test.shape == reference.shape
    scale = np.max(np.abs(reference))
    error = np.max(np.abs(test - reference)) / scale if scale > 0 else np.max(np.abs(test))
    aa = np.vdot(test, test).real
    bb = np.vdot(reference, reference).real
    mismatch = 0.0 if aa == 0 and bb == 0 else 1.0 - np.vdot(reference, test).real / np.sqrt(aa * bb)
    return error, mismatch


@pytest.fixture(scope="session")
def cuda():
    """The CUDA device, or skip (the ``gpu`` tests only run where one is)."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
