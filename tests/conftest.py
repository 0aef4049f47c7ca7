"""Shared test configuration: the ``gpu`` marker and fixture loading."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
for p in (str(ROOT),):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libfitb200.so")


def load_golden(name: str):
    """Problem and reference outputs of one fixture."""
    from magnelio_b200.problem import FitProblem

    d = dict(np.load(GOLDEN / f"{name}.npz", allow_pickle=False))
    return FitProblem.from_arrays(d), d, int(d["n_steps"])


@pytest.fixture
def golden():
    return load_golden
