"""Shared set-up: import paths, the ``gpu`` marker and the oracle fixtures.

Tests marked ``gpu`` need a B200 and run with ``pytest -m gpu``; everything
else runs on a CPU-only machine.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "asd-kernel-fusion_b200"
GOLDEN = ROOT / "tests" / "golden"
for p in (PKG, ROOT / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")


@pytest.fixture(scope="session")
def oracle():
    import oracle as orc

    lib = orc.HERE / "liboracle.so"
    if not lib.exists():
        orc.build()
    return orc.Oracle()


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return dict(np.load(GOLDEN / f"{name}.npz"))

    return load


def rel_err(a: complex, b: complex) -> float:
    return abs(a - b) / max(abs(b), 1e-300)
