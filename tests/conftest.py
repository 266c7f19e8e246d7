"""Shared test setup: import paths and the ``gpu`` marker.

Tests marked ``gpu`` need a B200 and the built CUDA library; everything else
runs on the CPU (the C restatement of the step in oracle/ is the checker).
"""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT / "gamera-op_b200", ROOT / "oracle", ROOT):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

GOLDEN = ROOT / "tests" / "golden"
NG = 4


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def load_golden(name):
    z = np.load(GOLDEN / f"{name}.npz", allow_pickle=False)
    return {k: z[k] for k in z.files}


def active(n):
    """Slices of the active cells plus the upper face on every axis."""
    return tuple(slice(NG, NG + m + 1) for m in n)


def rel_l1(a, b):
    den = np.abs(b).sum()
    return float(np.abs(a - b).sum() / den) if den > 0 else float(np.abs(a - b).sum())


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.lib()
    return oracle
