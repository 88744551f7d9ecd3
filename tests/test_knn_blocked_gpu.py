"""kNN when the distance column does not fit the allowed device memory: rows
are computed in blocks against every column and ranked per block (the
reference's sparseDists works in chunks too, src/gpu/dist.cu:495-791).  The
blocked results must be identical to the one-column results: same neighbours,
same order, same float distances."""
import numpy as np
import pytest

from conftest import random_sketches
from sketchlib_b200 import capi

pytestmark = pytest.mark.gpu

LIMIT = 300_000          # bytes: 900 samples -> 256-row blocks


@pytest.fixture
def ctx(gpu_ctx):
    yield gpu_ctx
    gpu_ctx.set_memory_limit(0)
    gpu_ctx.set_semantics(capi.SEMANTICS_REFERENCE_CPU)


def _both(ctx, fn):
    want = fn()
    ctx.set_memory_limit(LIMIT)
    try:
        got = fn()
    finally:
        ctx.set_memory_limit(0)
    for a, b in zip(got, want):
        np.testing.assert_array_equal(a, b)
    return want


@pytest.mark.parametrize("kind", ["none", "table", "equal_base"])
@pytest.mark.parametrize("semantics", [capi.SEMANTICS_REFERENCE_CPU, capi.SEMANTICS_REFERENCE_GPU])
def test_self_knn_blocked(ctx, kind, semantics):
    """The Monte Carlo table is asymmetric in its clusters: a block that saw
    a pair as (larger index, smaller index) must still read the entry the
    all-vs-all path reads."""
    n, K, s64 = 900, 4, 16
    words, kmers = random_sketches(n, K, s64, seed=1301)
    rng = np.random.default_rng(7)
    cl = rng.integers(0, 3, n).astype(np.uint16)
    lens = rng.integers(1_000_000, 5_000_000, n).astype(np.uint64)
    table = rng.uniform(0, 0.02, (K, 3, 3)).astype(np.float32)
    rnd = {"none": None,
           "table": capi.Random(ctx, capi.RANDOM_TABLE, kmers, table=table),
           "equal_base": capi.Random(ctx, capi.RANDOM_EQUAL_BASE, kmers)}[kind]
    ctx.set_semantics(semantics)
    db = capi.Database(ctx, words, kmers, s64, cluster=cl, seq_len=lens)
    for col in (0, 1):
        _both(ctx, lambda: capi.dists_knn(ctx, db, 7, dist_col=col, random=rnd))
    _both(ctx, lambda: capi.dists_knn(ctx, db, 5, dist_col=1, jaccard=True, random=rnd))


def test_self_knn_blocked_all_neighbours(ctx):
    """kNN = n ranks every column, the sample's own (+inf) last."""
    words, kmers = random_sketches(300, 3, 8, seed=1302)
    db = capi.Database(ctx, words, kmers, 8)
    want = capi.dists_knn(ctx, db, 300)
    ctx.set_memory_limit(100_000)                        # 300 samples -> 256-row blocks
    got = capi.dists_knn(ctx, db, 300)
    for a, b in zip(got, want):
        np.testing.assert_array_equal(a, b)
    assert np.isinf(want[2].reshape(300, 300)[:, -1]).all()


def test_query_knn_blocked(ctx):
    words, kmers = random_sketches(1300, 4, 16, seed=1303)
    ref = capi.Database(ctx, words[:700], kmers, 16)
    qry = capi.Database(ctx, words[700:], kmers, 16)
    _both(ctx, lambda: capi.query_knn(ctx, ref, qry, 9, dist_col=0))
