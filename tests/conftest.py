"""Shared fixtures.  Tests marked ``gpu`` need a CUDA device; everything else
runs on a CPU-only machine (oracle, host logic, library loading)."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "rust-nmf_b200"
for path in (str(ROOT), str(PKG)):
    if path not in sys.path:
        sys.path.insert(0, path)

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def quickstart():
    """V, W0, H0 of the reference's quickstart notebook."""
    z = np.load(GOLDEN / "quickstart_inputs.npz")
    return z["V"], z["W0"], z["H0"]


@pytest.fixture(scope="session")
def kats():
    return json.loads((GOLDEN / "quickstart_kats.json").read_text())


@pytest.fixture(scope="session")
def oracle():
    import oracle as orc

    orc.build()
    return orc


def rel_max(a: np.ndarray, b: np.ndarray) -> float:
    """max|a - b| / max|b| -- the parity measure of the factors."""
    scale = float(np.max(np.abs(b))) if b.size else 0.0
    return float(np.max(np.abs(a - b))) / (scale if scale > 0 else 1.0)


def rel(a: float, b: float) -> float:
    return abs(a - b) / max(abs(b), 1e-300)
