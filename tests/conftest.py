"""Test configuration: the ``gpu`` marker and shared fixtures.

``-m "not gpu"`` runs the oracle pins, host logic and C-ABI load checks on
any machine; ``-m gpu`` runs the parity tests through the C ABI on a CUDA
device.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(scope="session")
def golden():
    def load(name):
        with np.load(GOLDEN / name, allow_pickle=False) as data:
            return {k: data[k] for k in data.files}
    return load


def case_from_golden(g, prefix="case"):
    """Rebuild a case dict from the arrays stored by make_golden.py."""
    from string_vext_b200.synth import make_case
    cell = g[f"{prefix}_cell"]
    lengths = np.linalg.norm(cell, axis=1)
    a, b, c = cell
    angles = np.degrees([np.arccos(b @ c / (lengths[1] * lengths[2])),
                         np.arccos(a @ c / (lengths[0] * lengths[2])),
                         np.arccos(a @ b / (lengths[0] * lengths[1]))])
    eps, sig, bond = g[f"{prefix}_guest"]
    case = make_case(lengths, angles, g[f"{prefix}_frac"], g[f"{prefix}_sigma"],
                     g[f"{prefix}_epsilon"], (eps, sig, bond), float(g[f"{prefix}_cutoff"]))
    case["cell"] = cell          # exactly the stored matrix
    return case
