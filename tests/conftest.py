"""Shared test setup: the `gpu` marker, repository paths, and the oracle import path.

Tests marked `gpu` need a CUDA device and call the product through the C-ABI
(libhippolbm.so); every other test runs on the CPU.  The oracle (oracle/) is test
infrastructure: it is imported here only as the checker.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")
DECKS = os.path.join(GOLDEN, "decks")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libhippolbm.so")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    if not oracle.available("port"):
        oracle.build("port")
    return oracle


def per_population_rel_err(f, f_ref, mask=None):
    """max over populations of |f - f_ref| / |f_ref| (0 where both are 0), over the nodes of
    `mask` (a boolean node array, or None for all).  Arrays are (19, nodes...); compared one
    direction at a time so that lattices of billions of values need no full-size temporaries."""
    import numpy as np

    worst = 0.0
    for i in range(f.shape[0]):
        a = np.asarray(f[i], dtype=np.float64)
        b = np.asarray(f_ref[i], dtype=np.float64)
        if mask is not None:
            a, b = a[mask], b[mask]
        d = np.abs(a - b)
        den = np.abs(b)
        bad = (d > 0) & (den == 0)
        if bad.any():
            return float("inf")
        with np.errstate(divide="ignore", invalid="ignore"):
            r = np.where(den > 0, d / np.where(den > 0, den, 1.0), 0.0)
        worst = max(worst, float(r.max()) if r.size else 0.0)
    return worst


def cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)
