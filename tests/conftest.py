"""Shared pytest configuration: the ``gpu`` marker and golden-fixture loading."""

from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a) and the built CUDA library")


def load_golden(name: str):
    """Return (arrays, params) for one committed golden fixture."""
    data = np.load(GOLDEN / f"{name}.npz", allow_pickle=False)
    arrays = {key: data[key] for key in data.files if key != "params_json"}
    params = json.loads(str(data["params_json"]))
    return arrays, params


def golden_vrows(arrays):
    """Group the reference's weighted contraction rows by K from a solve fixture."""
    groups, B_real, B_imag = {}, {}, {}
    for key, value in arrays.items():
        if key.startswith("vrows_idx_"):
            K = int(key.rsplit("_", 1)[1])
            groups[K] = tuple(int(i) for i in value)
            B_real[K] = arrays[f"vrows_real_{K}"]
            if f"vrows_imag_{K}" in arrays:
                B_imag[K] = arrays[f"vrows_imag_{K}"]
    return groups, B_real, (B_imag or None), float(arrays["vrows_norm"])


@pytest.fixture
def golden():
    return load_golden
