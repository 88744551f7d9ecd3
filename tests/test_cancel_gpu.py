"""Cancellation, the failure this library can inject without faulting a GPU:
another thread sets the context's mapped cancel word while a long all-vs-all
runs (what the drop-in module does on Ctrl-C, where the reference trapped the
kernel, src/gpu/cuda.cuh:77-87).  The kernels stop fetching work, end their
stream through the normal end-of-work step, and the call reports
SK_ECANCELLED; the context then computes correctly again."""
import threading
import time

import numpy as np
import pytest

import oracle
from conftest import random_sketches
from sketchlib_b200 import capi

pytestmark = pytest.mark.gpu


def test_cancel_running_all_vs_all_then_reuse(gpu_ctx):
    import torch
    from sketchlib_b200 import synth
    n, kmers, s64 = 16_384, list(range(15, 31, 2)), 156
    parent, thresh = synth.random_tree(n, kmers=kmers, seed=0x5EEDCA11)
    words = torch.empty(n * len(kmers) * s64 * 14, dtype=torch.int64, device="cuda")
    capi.synth_device(gpu_ctx, parent, thresh, s64, seed=0x5EEDCA11, d_words=words.data_ptr())
    db = capi.Database(gpu_ctx, words.data_ptr(), kmers, s64, n_samples=n)
    out = torch.empty((n * (n - 1) // 2, 2), dtype=torch.float32, device="cuda")
    capi.dists_dense(gpu_ctx, db, out=out.data_ptr())      # warm (about 0.3 s)
    gpu_ctx.synchronize()

    errors = []

    def run():
        try:
            capi.dists_dense(gpu_ctx, db, out=out.data_ptr())
            gpu_ctx.synchronize()
        except capi.SketchlibError as exc:
            errors.append(exc)

    th = threading.Thread(target=run)
    t0 = time.perf_counter()
    th.start()
    time.sleep(0.03)
    gpu_ctx.cancel()
    th.join(timeout=60)
    assert not th.is_alive()
    assert len(errors) == 1 and errors[0].status == capi.SK_ECANCELLED, errors
    assert time.perf_counter() - t0 < 5.0

    # the context is usable again, and a cancel issued before a call is ignored
    gpu_ctx.cancel()
    small, km = random_sketches(200, 4, 16, seed=77)
    sdb = capi.Database(gpu_ctx, small, km, 16)
    np.testing.assert_array_equal(capi.dists_dense(gpu_ctx, sdb, out_mode=capi.OUT_COUNTS),
                                  oracle.dists(small, km, 16, out_mode=2))
    sdb.close()
    db.close()
