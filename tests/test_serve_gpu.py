"""The query server: continuous batching over a resident reference database.
Each request's results must equal the direct query-vs-reference computation,
and be bit-identical whether the request runs alone or mixed with others."""
import threading

import numpy as np
import pytest

from conftest import random_sketches
from sketchlib_b200 import capi

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    ctx = capi.Context(0)
    n_ref, K, s64 = 1500, 8, 156
    words, kmers = random_sketches(n_ref + 700, K, s64, seed=33)
    ref = capi.Database(ctx, words[:n_ref], kmers, s64)
    queries = words[n_ref:]
    yield ctx, ref, queries, kmers
    ref.close()
    ctx.close()


def _expected(ctx, ref, q, kmers, knn):
    qdb = capi.Database(ctx, q, kmers, 156)
    rows = capi.dists_dense(ctx, ref, qdb).reshape(q.shape[0], ref.n, 2)
    idx, dist = capi.query_knn(ctx, ref, qdb, knn, dist_col=0)
    qdb.close()
    return rows, idx, dist


def test_alone_and_mixed_results_identical(setup):
    ctx, ref, queries, kmers = setup
    sizes = [1, 7, 130, 64, 300, 2, 180]
    offs = np.cumsum([0] + sizes)
    reqs = [queries[offs[i]:offs[i + 1]] for i in range(len(sizes))]
    server = capi.Server(ctx, ref, slots=3, slice_queries=64, kNN=5, keep_rows=True)
    try:
        alone = []
        for q in reqs:
            t = server.submit(q)
            server.wait(t)
            idx, dist, rows, lat = server.result(t)
            assert lat > 0
            e_rows, e_idx, e_dist = _expected(ctx, ref, q, kmers, 5)
            np.testing.assert_array_equal(rows, e_rows)
            np.testing.assert_array_equal(idx, e_idx)
            np.testing.assert_array_equal(dist, e_dist)
            alone.append((idx, dist, rows))
        # now everything at once, from several threads, plus repeats
        tickets = {}
        lock = threading.Lock()

        def submit(i):
            t = server.submit(reqs[i])
            with lock:
                tickets.setdefault(i, []).append(t)

        threads = [threading.Thread(target=submit, args=(i % len(reqs),))
                   for i in range(3 * len(reqs))]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        for i, ts in tickets.items():
            for t in ts:
                server.wait(t)
                idx, dist, rows, _ = server.result(t)
                np.testing.assert_array_equal(idx, alone[i][0])
                np.testing.assert_array_equal(dist, alone[i][1])
                np.testing.assert_array_equal(rows, alone[i][2])
        st = server.stats()
        assert st["queued_queries"] == 0 and st["pairs_done"] >= 4 * sum(sizes) * ref.n
    finally:
        server.close()


def test_server_wait_timeout_and_bad_ticket(setup):
    ctx, ref, queries, _ = setup
    server = capi.Server(ctx, ref, slots=1, slice_queries=32, kNN=3)
    try:
        with pytest.raises(capi.SketchlibError):
            server.wait(987654, timeout=0.1)
        t = server.submit(queries[:40])
        server.wait(t, timeout=30)
        idx, dist, rows, _ = server.result(t)
        assert rows is None and idx.shape == (40, 3)
        assert np.all(np.diff(dist, axis=1) >= 0)
    finally:
        server.close()


def test_server_keeps_the_context_semantics(setup):
    """A server created under the reference-GPU semantics answers with them."""
    ctx, ref, queries, kmers = setup
    q = queries[:40]
    ctx.set_semantics(capi.SEMANTICS_REFERENCE_GPU)
    try:
        e_rows, e_idx, e_dist = _expected(ctx, ref, q, kmers, 5)
        server = capi.Server(ctx, ref, slots=2, slice_queries=16, kNN=5, keep_rows=True)
    finally:
        ctx.set_semantics(capi.SEMANTICS_REFERENCE_CPU)
    try:
        t = server.submit(q)
        server.wait(t)
        idx, dist, rows, _ = server.result(t)
        np.testing.assert_array_equal(rows, e_rows)
        np.testing.assert_array_equal(idx, e_idx)
        np.testing.assert_array_equal(dist, e_dist)
        cpu_rows, _, _ = _expected(ctx, ref, q, kmers, 5)
        assert np.any(cpu_rows != rows)
    finally:
        server.close()


def test_priority_slicing_with_equal_base(setup):
    """Requests larger than slice_queries run in large_slice_queries slices
    (low priority, at most half the slots), the others as one high-priority
    slice; free slots go to the fewest queries left.  Under the equal-base
    random-match model with per-sample lengths, every result equals the direct
    query-vs-reference computation whatever order the scheduler chose."""
    ctx, _, queries, kmers = setup
    rng = np.random.default_rng(5)
    ref_words, q_words = queries[:500], queries[500:700]
    ref_len = rng.integers(1_000_000, 5_000_000, 500).astype(np.uint64)
    q_len = rng.integers(1_000_000, 5_000_000, 200).astype(np.uint64)
    ref = capi.Database(ctx, ref_words, kmers, 156, seq_len=ref_len)
    rnd = capi.Random(ctx, capi.RANDOM_EQUAL_BASE, kmers)
    with pytest.raises(capi.SketchlibError):
        capi.Server(ctx, ref, random=rnd, slots=2, slice_queries=16, kNN=3,
                    large_slice_queries=17)
    server = capi.Server(ctx, ref, random=rnd, slots=4, slice_queries=64, kNN=4,
                         keep_rows=True, large_slice_queries=24)
    try:
        sizes = [100, 3, 64, 1, 20, 12]
        offs = np.cumsum([0] + sizes)
        tickets = [server.submit(q_words[offs[i]:offs[i + 1]], seq_len=q_len[offs[i]:offs[i + 1]])
                   for i in range(len(sizes))]
        for i, t in enumerate(tickets):
            server.wait(t)
            idx, dist, rows, _ = server.result(t)
            q = q_words[offs[i]:offs[i + 1]]
            qdb = capi.Database(ctx, q, kmers, 156, seq_len=q_len[offs[i]:offs[i + 1]])
            e_rows = capi.dists_dense(ctx, ref, qdb, random=rnd).reshape(len(q), ref.n, 2)
            e_idx, e_dist = capi.query_knn(ctx, ref, qdb, 4, dist_col=0, random=rnd)
            qdb.close()
            np.testing.assert_array_equal(rows, e_rows)
            np.testing.assert_array_equal(idx, e_idx)
            np.testing.assert_array_equal(dist, e_dist)
    finally:
        server.close()
        rnd.close()
        ref.close()
