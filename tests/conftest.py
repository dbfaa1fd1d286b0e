"""Shared test set-up.

* Registers the ``gpu`` marker: tests that need a B200 (``-m gpu``).
* Puts the product package (``particle-simulator_b200``, which holds the
  drop-in ``dem`` package) and the oracle on ``sys.path``.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "particle-simulator_b200"
for p in (str(PKG), str(ROOT / "oracle"), str(ROOT)):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return dict(np.load(GOLDEN / name, allow_pickle=False))

    return load


@pytest.fixture(scope="session")
def cuda_available():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False
