"""The device-side bounded wait: a kernel waiting on a barrier that nothing
completes gives up after its limit and reports it (SK_ETIMEDOUT), with no
fault, trap or endless spin, and the context computes correctly afterwards.
Every wait in this library's kernels is this bounded wait."""
import time

import numpy as np
import pytest

import oracle
from conftest import random_sketches
from sketchlib_b200 import capi

pytestmark = pytest.mark.gpu


def test_wait_runs_out_and_context_stays_usable(gpu_ctx):
    t0 = time.perf_counter()
    st = capi.lib.sk_probe_wait_limit(gpu_ctx.handle, 200)
    elapsed = time.perf_counter() - t0
    assert st == capi.SK_ETIMEDOUT
    assert "bounded wait" in gpu_ctx.last_error
    assert 0.19 < elapsed < 5.0
    words, kmers = random_sketches(150, 3, 8, seed=91)
    db = capi.Database(gpu_ctx, words, kmers, 8)
    np.testing.assert_array_equal(capi.dists_dense(gpu_ctx, db, out_mode=capi.OUT_COUNTS),
                                  oracle.dists(words, kmers, 8, out_mode=2))
    db.close()


def test_wait_limit_arguments(gpu_ctx):
    assert capi.lib.sk_probe_wait_limit(gpu_ctx.handle, 0) == capi.SK_EINVAL
    assert capi.lib.sk_probe_wait_limit(gpu_ctx.handle, 20_000) == capi.SK_EINVAL
