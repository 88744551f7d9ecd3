"""Shared test setup: import paths, the gpu marker, seeded sketch fixtures."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT, ROOT / "pp-sketchlib_b200", ROOT / "oracle"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def random_sketches(n, K, s64, seed, related=True):
    """Seeded synthetic sketches in the reference word layout."""
    from sketchlib_b200 import synth, capi
    kmers = list(range(15, 15 + 2 * K, 2))
    if related:
        parent, thresh = synth.random_tree(n, kmers=kmers, seed=seed)
        words = capi.synth_host(parent, thresh, s64, seed=seed, threads=8)
    else:
        rng = np.random.default_rng(seed)
        words = rng.integers(0, 2 ** 64, size=(n, K, s64 * 14), dtype=np.uint64)
    return words, np.asarray(kmers, dtype=np.int32)


@pytest.fixture(scope="session")
def gpu_ctx():
    from sketchlib_b200 import capi
    ctx = capi.Context(0)
    yield ctx
    ctx.close()
