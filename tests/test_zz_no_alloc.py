"""sk_dists_dense_noalloc: dense distances with no device allocation.

Callers that cannot allocate device memory when they ask for distances (a
service whose device memory is partitioned at start-up, a host sharing the
GPU with an allocator it does not control) use this entry point; its scratch is a static device buffer inside the
library.  Checked here through the C ABI against the allocating entry point,
sk_dists_dense, on two calls in a row, with the tolerances of the parity tests
(counts and Jaccard exact, core/accessory 1e-6).  The file is named to be
collected last and makes its own context, so it passes alone or after the
other tests.
"""
import numpy as np
import pytest

from conftest import random_sketches
from sketchlib_b200 import capi

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _noalloc(ctx, ref, query, rnd, mode, out):
    st = capi.lib.sk_dists_dense_noalloc(ctx.handle, ref.handle,
                                          None if query is None else query.handle,
                                          None if rnd is None else rnd.handle, mode, out.data_ptr())
    assert st == capi.SK_OK, ctx.last_error
    ctx.synchronize()


@pytest.mark.parametrize("case", ["self_coreacc", "query_equal_base", "self_table_jaccard",
                                  "self_counts", "query_table", "self_equal_base_refgpu"])
def test_noalloc_matches_allocating_entry_point(case):
    import torch
    ctx = capi.Context(0)
    n, nq, K, s64 = 700, 90, 8, 156
    w, kmers = random_sketches(n + nq, K, s64, seed=7)
    rng = np.random.default_rng(7)
    lens = rng.integers(1_000_000, 6_000_000, n + nq).astype(np.uint64)
    cl = rng.integers(0, 3, n + nq).astype(np.uint16)
    kmers = np.arange(11, 11 + 2 * K, 2, dtype=np.int32)
    ref = capi.Database(ctx, w[:n], kmers, s64, cluster=cl[:n], seq_len=lens[:n])
    qry = capi.Database(ctx, w[n:], kmers, s64, cluster=cl[n:], seq_len=lens[n:])
    query, rnd, mode = None, None, capi.OUT_CORE_ACC
    if case == "query_equal_base":
        query = qry
        rnd = capi.Random(ctx, capi.RANDOM_EQUAL_BASE, kmers)
    elif case == "self_table_jaccard":
        rnd = capi.Random(ctx, capi.RANDOM_TABLE, kmers,
                          table=rng.uniform(0, 0.01, (K, 3, 3)).astype(np.float32))
        mode = capi.OUT_JACCARD
    elif case == "self_counts":
        mode = capi.OUT_COUNTS
    elif case == "query_table":
        query = qry
        rnd = capi.Random(ctx, capi.RANDOM_TABLE, kmers,
                          table=rng.uniform(0, 0.01, (K, 3, 3)).astype(np.float32))
    elif case == "self_equal_base_refgpu":
        # the reference GPU path's equal-base branch: one chance per k from
        # the first reference's length
        ctx.set_semantics(capi.SEMANTICS_REFERENCE_GPU)
        rnd = capi.Random(ctx, capi.RANDOM_EQUAL_BASE, kmers)
    want = capi.dists_dense(ctx, ref, query, rnd, out_mode=mode)
    dtype = torch.int32 if mode == capi.OUT_COUNTS else torch.float32
    out = torch.empty(want.shape, dtype=dtype, device="cuda")
    for _ in range(2):                    # two calls in a row share the static buffer
        out.fill_(-1)
        _noalloc(ctx, ref, query, rnd, mode, out)
        got = out.cpu().numpy()
        if mode == capi.OUT_CORE_ACC:
            np.testing.assert_allclose(got, want, atol=TOL, rtol=0)
        elif mode == capi.OUT_COUNTS:
            np.testing.assert_array_equal(got.view(np.uint32), want)
        else:
            np.testing.assert_array_equal(got, want)
    ctx.close()


def test_noalloc_rejects_jobs_beyond_its_buffer():
    """A job whose equal-base random-match factors alone exceed the static
    buffer (262,145 references x 32 k-mer lengths of doubles) is refused
    before anything is launched.  The output buffer is still full size, so the
    call could not write out of bounds even if it ran."""
    import torch
    from sketchlib_b200 import synth
    ctx = capi.Context(0)
    n, K, s64 = 262_145, 32, 1
    kmers = list(range(5, 5 + K))
    parent, thresh = synth.random_tree(n, kmers=kmers, seed=3)
    words = torch.empty(n * K * s64 * 14, dtype=torch.int64, device="cuda")
    capi.synth_device(ctx, parent, thresh, s64, seed=3, d_words=words.data_ptr())
    ref = capi.Database(ctx, words.data_ptr(), kmers, s64, n_samples=n,
                        seq_len=np.full(n, 3_000_000, np.uint64))
    qry = capi.Database(ctx, words.data_ptr(), kmers, s64, n_samples=1,
                        seq_len=np.full(1, 3_000_000, np.uint64))
    del words
    rnd = capi.Random(ctx, capi.RANDOM_EQUAL_BASE, kmers)
    out = torch.empty((capi.dists_rows(ref, qry), 2), dtype=torch.float32, device="cuda")
    st = capi.lib.sk_dists_dense_noalloc(ctx.handle, ref.handle, qry.handle, rnd.handle,
                                          capi.OUT_CORE_ACC, out.data_ptr())
    assert st == 9, ctx.last_error   # SK_ERANGE
    assert "static" in ctx.last_error and "sk_dists_dense" in ctx.last_error
    ctx.close()
