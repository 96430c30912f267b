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
