"""Shared test setup: import paths, the `gpu` marker, seeded helpers."""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "qpg-rotormap_b200"))
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


def pytest_collection_modifyitems(config, items):
    # keep the marker honest: a gpu test on a machine without CUDA is skipped
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:  # pragma: no cover
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def random_words(rng, n, k):
    """n fragments of k random bases, forward-packed with a zero tail."""
    W = (k + 15) // 16
    w = rng.integers(0, 2 ** 32, size=(n, W), dtype=np.uint64).astype(np.uint32)
    r = k & 15
    if r:
        w[:, -1] &= np.uint32((1 << (2 * r)) - 1)
    return w


@pytest.fixture
def rng():
    return np.random.default_rng(1234)
