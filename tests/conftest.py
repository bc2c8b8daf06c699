"""Shared pytest configuration: the `gpu` marker and common helpers."""

from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long-running test")


def _has_cuda() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:  # noqa: BLE001
        return False


def pytest_collection_modifyitems(config, items):
    if _has_cuda():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def load_golden(name: str) -> dict:
    data = np.load(GOLDEN / name, allow_pickle=False)
    out: dict = {}
    for k in data.files:
        if "/" in k:
            p, r = k.split("/")
            out.setdefault(int(p), {})[r] = data[k]
        else:
            out[k] = data[k]
    return out


def rel_err(a, b) -> float:
    """max |a-b| / max(1, |b|) over entries finite in both; inf if the
    non-finite patterns differ."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    fa, fb = np.isfinite(a), np.isfinite(b)
    if not np.array_equal(fa, fb):
        return float("inf")
    if not np.array_equal(np.where(fa, 0, a), np.where(fb, 0, b), equal_nan=True):
        return float("inf")
    if not fa.any():
        return 0.0
    d = np.abs(a[fa] - b[fa]) / np.maximum(1.0, np.abs(b[fa]))
    return float(d.max())
