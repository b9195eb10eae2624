"""Test set-up: the repository root on sys.path, the ``gpu`` marker, and the golden fixtures.

Tests marked ``gpu`` need a B200 and call the CUDA library through its C ABI; the rest run on the
CPU: the oracle against the golden fixtures and the reference, the host logic, and the library's
exports (no compute without a GPU).
"""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
for path in (ROOT, ROOT / "tests"):
    if str(path) not in sys.path:
        sys.path.insert(0, str(path))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (CUDA sm_100a) and the built library")


def golden_names() -> list[str]:
    return list(json.loads((GOLDEN / "manifest.json").read_text()))


def still_names() -> list[str]:
    """The golden grids without moving air: the ones the compensated form and stacking take."""
    return [n for n in golden_names() if not n.startswith("wind_")]


def load_golden(name: str):
    """(layout, signal, reference) of a golden fixture: the reference's layout arrays, the drive,
    and the reference's own probe series (probes, steps)."""
    with np.load(GOLDEN / f"{name}.npz") as data:
        layout = {k.split("/", 1)[1]: data[k] for k in data.files if k.startswith("layout/")}
        return layout, data["signal"], data["reference"]
