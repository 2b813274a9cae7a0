"""Shared fixtures: golden-vector loading and tolerance helpers."""

import sys
from pathlib import Path
from types import SimpleNamespace

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
GOLDEN = REPO / "tests" / "golden"
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100a) and the built CUDA library")


def golden(name):
    return np.load(GOLDEN / f"{name}.npz")


def cfg_from(d, prefix="cfg_", cls=None):
    """Rebuild an OpticalConfig (or a namespace) from a fixture's cfg_* fields."""
    kw = {}
    for k in d.files:
        if k.startswith(prefix):
            v = d[k]
            kw[k[len(prefix):]] = tuple(v.tolist()) if v.ndim else v.item()
    if cls is None:
        from maomi_b200.optics import OpticalConfig as cls
    return cls(**kw)


def rel_l2(actual, expected):
    a = np.asarray(actual)
    b = np.asarray(expected)
    a = a.astype(np.complex128 if np.iscomplexobj(a) else np.float64)
    b = b.astype(np.complex128 if np.iscomplexobj(b) else np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


@pytest.fixture
def ns():
    return SimpleNamespace
