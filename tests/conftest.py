"""Shared pytest configuration: the ``gpu`` marker, repo paths and golden cases."""
from __future__ import annotations

import json
import pathlib
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
PKG = ROOT / "factor-cuda_b200"
for p in (str(ROOT), str(PKG)):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    """(cases, arrays) of tests/golden/golden_v1.*"""
    meta = json.loads((GOLDEN / "golden_v1.json").read_text())
    arrays = dict(np.load(GOLDEN / "golden_v1.npz"))
    return meta["cases"], arrays


def bitwise_f32(a, b):
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    return a.shape == b.shape and bool(np.array_equal(a.view(np.uint32), b.view(np.uint32)))


def corr_match(a, b, tol=1e-12):
    """NaN / inf pattern equality plus |a-b| <= tol on finite cells (the
    reference suite's rule, tests/test_adapter_v1.py:67-82)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if a.shape != b.shape:
        return False
    if not np.array_equal(np.isnan(a), np.isnan(b)):
        return False
    if not np.array_equal(np.isposinf(a), np.isposinf(b)):
        return False
    if not np.array_equal(np.isneginf(a), np.isneginf(b)):
        return False
    fin = np.isfinite(a) & np.isfinite(b)
    return bool(np.all(np.abs(a[fin] - b[fin]) <= tol))
