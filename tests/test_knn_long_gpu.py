"""kNN lists longer than the per-lane shared-memory lists (kNN > 800): radix
select and a bitonic sort per dense row.  Self lists are checked against the
oracle's restatement of query_db_sparse (src/api.cpp:332-432) on the GPU's own
dense values, query lists against a stable argsort of the dense rows (the
reference test's check), both exactly: same neighbours, same order (ties by
the smaller index), same floats.  Short sketches (sketchsize64 2 and 4) make
many exactly equal distances, so the tie rule is exercised at the cut."""
import numpy as np
import pytest

import oracle
from conftest import random_sketches
from sketchlib_b200 import capi

pytestmark = pytest.mark.gpu


@pytest.fixture
def ctx(gpu_ctx):
    yield gpu_ctx
    gpu_ctx.set_memory_limit(0)


def _self_case(ctx, n, K, s64, seed):
    words, kmers = random_sketches(n, K, s64, seed=seed)
    words[5] = words[6]              # exact ties at distance 0
    words[7] = words[6]
    return words, kmers, capi.Database(ctx, words, kmers, s64)


@pytest.mark.parametrize("knn", [801, 1000, 1100])
@pytest.mark.parametrize("jaccard,dist_col", [(False, 0), (False, 1), (True, 1)])
def test_self_knn_long_lists(ctx, knn, jaccard, dist_col):
    n, K, s64 = 1100, 3, 4
    words, kmers, db = _self_case(ctx, n, K, s64, seed=2001 + knn)
    i, j, d = capi.dists_knn(ctx, db, knn, dist_col=dist_col, jaccard=jaccard)
    if jaccard:
        dense = capi.dists_dense(ctx, db, out_mode=capi.OUT_JACCARD)
        oi, oj, od = oracle.knn_self(dense, n, dist_col, knn, jaccard_=True)
    else:
        dense = capi.dists_dense(ctx, db)
        oi, oj, od = oracle.knn_self(dense, n, dist_col, knn)
    np.testing.assert_array_equal(i, oi)
    np.testing.assert_array_equal(j, oj)
    np.testing.assert_array_equal(d, od)
    if knn == n:                     # every column ranked, the sample's own (+inf) last
        assert np.all(j.reshape(n, knn)[:, -1] == np.arange(n))


def test_self_knn_long_lists_in_blocks(ctx):
    """The same lists when the rows are computed in blocks of 256 (the
    allowed memory holds fewer rows than the database has)."""
    n, K, s64, knn = 1100, 3, 4, 900
    _, _, db = _self_case(ctx, n, K, s64, seed=2011)
    want = capi.dists_knn(ctx, db, knn, dist_col=0)
    ctx.set_memory_limit(1_200_000)
    got = capi.dists_knn(ctx, db, knn, dist_col=0)
    for a, b in zip(got, want):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("nr,knn,s64", [(4000, 3000, 2),    # list sorted in shared memory
                                        (13000, 12500, 2),  # list sorted in its output slots
                                        (2500, 2500, 4)])   # every reference ranked
def test_query_knn_long_lists(ctx, nr, knn, s64):
    nq, K = 24, 3
    rw, kmers = random_sketches(nr, K, s64, seed=2021 + nr)
    qw = rw[:nq].copy()              # queries identical to some references
    ref = capi.Database(ctx, rw, kmers, s64)
    qry = capi.Database(ctx, qw, kmers, s64)
    for col in (0, 1):
        r, d = capi.query_knn(ctx, ref, qry, knn, dist_col=col)
        dense = capi.dists_dense(ctx, ref, qry)[:, col].reshape(nq, nr)
        order = np.argsort(dense, axis=1, kind="stable")[:, :knn]
        np.testing.assert_array_equal(r, order)
        np.testing.assert_array_equal(d, np.take_along_axis(dense, order, axis=1))


def test_query_knn_long_list_matches_short_list_prefix(ctx):
    """A long list starts with the short list of the shared-memory kernel."""
    nr, nq, K, s64 = 3000, 40, 4, 16
    rw, kmers = random_sketches(nr, K, s64, seed=2031)
    ref = capi.Database(ctx, rw, kmers, s64)
    qry = capi.Database(ctx, rw[100:100 + nq].copy(), kmers, s64)
    r_short, d_short = capi.query_knn(ctx, ref, qry, 800, dist_col=1)
    r_long, d_long = capi.query_knn(ctx, ref, qry, 2000, dist_col=1)
    np.testing.assert_array_equal(r_long[:, :800], r_short)
    np.testing.assert_array_equal(d_long[:, :800], d_short)
