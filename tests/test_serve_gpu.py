"""The query server: continuous batching over a resident reference database.

Every request's rows and top-kNN lists are checked against the CPU oracle
(the reference's query_db semantics, src/api.cpp:223-283, with the per-query
random-match inputs the request carried), and must be bit-identical whether
the request runs alone or packed into slices with others."""
import threading

import numpy as np
import pytest

import oracle
from conftest import random_sketches
from sketchlib_b200 import capi

pytestmark = pytest.mark.gpu

S64 = 156


@pytest.fixture(scope="module")
def setup():
    ctx = capi.Context(0)
    n_ref, K = 1200, 8
    words, kmers = random_sketches(n_ref + 700, K, S64, seed=33)
    ref = capi.Database(ctx, words[:n_ref], kmers, S64)
    yield ctx, ref, words[:n_ref], words[n_ref:], kmers
    ref.close()
    ctx.close()


def oracle_expected(ref_words, q, kmers, knn, random=None, dist_col=0):
    """Rows [n_q][n_ref][2] and the kNN lists (ascending, ties by smaller
    reference index) from the oracle's query-vs-reference distances."""
    rows = oracle.dists(ref_words, kmers, S64, query_words=q, random=random)
    rows = rows.reshape(q.shape[0], ref_words.shape[0], 2)
    d = rows[:, :, dist_col]
    j = np.arange(d.shape[1])
    idx = np.stack([np.lexsort((j, d[i]))[:knn] for i in range(d.shape[0])]).astype(np.int64)
    return rows, idx, np.take_along_axis(d, idx, axis=1)


def check(got, want, exact_rows=False):
    idx, dist, rows = got
    w_rows, w_idx, w_dist = want
    # the oracle's double fit and CUDA's log/exp may differ in the last ulp
    np.testing.assert_allclose(rows, w_rows, rtol=0, atol=1e-6)
    np.testing.assert_allclose(dist, w_dist, rtol=0, atol=1e-6)
    # a kNN list can only differ where two distances sit within that ulp
    bad = idx != w_idx
    if bad.any():
        d_got = np.take_along_axis(w_rows[:, :, 0], idx, axis=1)
        np.testing.assert_allclose(d_got[bad], w_dist[bad], rtol=0, atol=1e-6)


def test_alone_and_mixed_equal_and_match_the_oracle(setup):
    ctx, ref, ref_words, queries, kmers = setup
    sizes = [1, 7, 130, 64, 300, 2, 180]
    offs = np.cumsum([0] + sizes)
    reqs = [queries[offs[i]:offs[i + 1]] for i in range(len(sizes))]
    want = oracle_expected(ref_words, queries[:offs[-1]], kmers, 5)
    server = capi.Server(ctx, ref, slots=3, slice_queries=64, kNN=5, keep_rows=True)
    try:
        alone = []
        for i, q in enumerate(reqs):
            t = server.submit(q)
            server.wait(t)
            idx, dist, rows, lat = server.result(t)
            assert lat > 0
            sl = slice(offs[i], offs[i + 1])
            check((idx, dist, rows), (want[0][sl], want[1][sl], want[2][sl]))
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


def test_small_requests_share_slices(setup):
    """Requests that wait while the device is busy are packed into shared
    slices; each one's results equal the oracle's and its results alone."""
    ctx, ref, ref_words, queries, kmers = setup
    rng = np.random.default_rng(8)
    sizes = rng.integers(1, 9, 40)
    offs = np.cumsum(np.concatenate([[0], sizes]))
    want = oracle_expected(ref_words, queries[:offs[-1]], kmers, 4)
    server = capi.Server(ctx, ref, slots=2, slice_queries=64, kNN=4, keep_rows=True)
    try:
        big = server.submit(queries[400:700])      # keeps the device busy
        ts = [server.submit(queries[offs[i]:offs[i + 1]]) for i in range(len(sizes))]
        server.wait(big)
        server.result(big)
        mixed = []
        for i, t in enumerate(ts):
            server.wait(t)
            got = server.result(t)[:3]
            sl = slice(offs[i], offs[i + 1])
            check(got, (want[0][sl], want[1][sl], want[2][sl]))
            mixed.append(got)
        info = server.info()
        assert info["slices_shared"] >= 1
        assert info["slices"] <= 5 + len(sizes) // 2
        for i in (0, 17, 39):
            t = server.submit(queries[offs[i]:offs[i + 1]])
            server.wait(t)
            got = server.result(t)[:3]
            for a, b in zip(got, mixed[i]):
                np.testing.assert_array_equal(a, b)
    finally:
        server.close()


def _mc_model(ctx, kmers, n_clusters=3, seed=4):
    rng = np.random.default_rng(seed)
    table = rng.uniform(0.0, 0.02, (len(kmers), n_clusters, n_clusters)).astype(np.float32)
    table[len(kmers) // 2:] = 0.0
    rnd = capi.Random(ctx, capi.RANDOM_TABLE, kmers, table=table)
    return rnd, table


def test_monte_carlo_clusters_are_set_per_slice(setup):
    """A request without cluster ids that follows one with cluster ids on the
    same slot gets cluster 0, not the previous request's ids."""
    ctx, _, ref_words, queries, kmers = setup
    rng = np.random.default_rng(6)
    ref_cl = rng.integers(0, 3, ref_words.shape[0]).astype(np.uint16)
    ref = capi.Database(ctx, ref_words, kmers, S64, cluster=ref_cl)
    rnd, table = _mc_model(ctx, kmers)
    server = capi.Server(ctx, ref, random=rnd, slots=1, slice_queries=64, kNN=5, keep_rows=True)
    try:
        q = queries[:50]
        given = np.full(50, 2, np.uint16)
        t = server.submit(q, cluster=given)
        server.wait(t)
        got_given = server.result(t)[:3]
        t = server.submit(q)
        server.wait(t)
        got_none = server.result(t)[:3]
        for cl, got in ((given, got_given), (np.zeros(50, np.uint16), got_none)):
            spec = oracle.RandomSpec(mode=2, table=table, cl_rows=cl, cl_cols=ref_cl)
            check(got, oracle_expected(ref_words, q, kmers, 5, random=spec))
        assert np.any(got_given[2] != got_none[2])
    finally:
        server.close()
        rnd.close()
        ref.close()


def test_queries_get_the_nearest_centroid(setup):
    """Under a table model with centroids, queries submitted with a base
    composition and no cluster id take the nearest centroid's cluster
    (RandomMC::lookup_array -> closest_cluster), as the oracle assigns it."""
    ctx, _, ref_words, queries, kmers = setup
    rng = np.random.default_rng(9)
    ref_cl = rng.integers(0, 3, ref_words.shape[0]).astype(np.uint16)
    ref = capi.Database(ctx, ref_words, kmers, S64, cluster=ref_cl)
    rnd, table = _mc_model(ctx, kmers, seed=5)
    centroids = np.array([[0.3, 0.2, 0.2, 0.3], [0.2, 0.3, 0.3, 0.2], [0.35, 0.15, 0.15, 0.35]],
                         np.float32)
    rnd.set_centroids(centroids)
    server = capi.Server(ctx, ref, random=rnd, slots=2, slice_queries=64, kNN=5, keep_rows=True)
    try:
        q = queries[:90]
        bases = rng.dirichlet(np.ones(4) * 8, 90)
        t = server.submit(q, base_freq=bases)
        server.wait(t)
        got = server.result(t)[:3]
        cl = oracle.closest_cluster(centroids, bases, use_rc=True)
        assert len(np.unique(cl)) > 1
        spec = oracle.RandomSpec(mode=2, table=table, cl_rows=cl, cl_cols=ref_cl)
        check(got, oracle_expected(ref_words, q, kmers, 5, random=spec))
    finally:
        server.close()
        rnd.close()
        ref.close()


def test_slots_follow_the_memory_budget(setup):
    """With a device-memory budget the server makes as many slots as fit; a
    budget below one slot is refused, and queries wait for a slot's memory."""
    ctx, ref, ref_words, queries, kmers = setup
    probe = capi.Server(ctx, ref, slots=1, slice_queries=64, kNN=3)
    slot_bytes = probe.info()["slot_bytes"]
    probe.close()
    assert slot_bytes > 64 * ref.n * 4
    with pytest.raises(capi.SketchlibError) as e:
        capi.Server(ctx, ref, slots=4, slice_queries=64, kNN=3, device_bytes=slot_bytes // 2)
    assert e.value.status == capi.SK_ENOMEM
    server = capi.Server(ctx, ref, slots=8, slice_queries=64, kNN=3,
                         device_bytes=int(2.5 * slot_bytes))
    try:
        assert server.info()["slots"] == 2
    finally:
        server.close()
    server = capi.Server(ctx, ref, slots=8, slice_queries=64, kNN=3, large_slice_queries=32,
                         device_bytes=int(1.5 * slot_bytes))
    try:
        assert server.info()["slots"] == 1
        ts = [server.submit(queries[i * 200:(i + 1) * 200]) for i in range(3)]
        assert server.stats()["queued_queries"] >= 600 - 4 * 32
        for i, t in enumerate(ts):
            server.wait(t)
            idx, dist, _, _ = server.result(t)
            _, w_idx, w_dist = oracle_expected(ref_words, queries[i * 200:(i + 1) * 200], kmers, 3)
            np.testing.assert_allclose(dist, w_dist, rtol=0, atol=1e-6)
    finally:
        server.close()


def test_server_wait_timeout_and_bad_ticket(setup):
    ctx, ref, _, queries, _ = setup
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
    ctx, ref, _, queries, kmers = setup
    q = queries[:40]

    def direct():
        qdb = capi.Database(ctx, q, kmers, S64)
        rows = capi.dists_dense(ctx, ref, qdb).reshape(q.shape[0], ref.n, 2)
        idx, dist = capi.query_knn(ctx, ref, qdb, 5, dist_col=0)
        qdb.close()
        return rows, idx, dist

    ctx.set_semantics(capi.SEMANTICS_REFERENCE_GPU)
    try:
        e_rows, e_idx, e_dist = direct()
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
        cpu_rows, _, _ = direct()
        assert np.any(cpu_rows != rows)
    finally:
        server.close()


def test_priority_slicing_with_equal_base(setup):
    """Requests larger than slice_queries run in large_slice_queries slices
    (low priority, at most half the slots), the others packed into
    high-priority slices; free slots go to the fewest queries left.  Under the
    equal-base random-match model with per-sample lengths, every result equals
    the oracle's whatever order the scheduler chose."""
    ctx, _, _, queries, kmers = setup
    rng = np.random.default_rng(5)
    ref_words, q_words = queries[:500], queries[500:700]
    ref_len = rng.integers(1_000_000, 5_000_000, 500).astype(np.uint64)
    q_len = rng.integers(1_000_000, 5_000_000, 200).astype(np.uint64)
    ref = capi.Database(ctx, ref_words, kmers, S64, seq_len=ref_len)
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
        spec = oracle.RandomSpec(mode=1, len_rows=q_len, len_cols=ref_len)
        want = oracle_expected(ref_words, q_words, kmers, 4, random=spec)
        for i, t in enumerate(tickets):
            server.wait(t)
            got = server.result(t)[:3]
            sl = slice(offs[i], offs[i + 1])
            check(got, (want[0][sl], want[1][sl], want[2][sl]))
    finally:
        server.close()
        rnd.close()
        ref.close()


def test_pinned_and_pageable_requests_agree(setup):
    """A request in page-locked memory is uploaded straight from it, a
    pageable one is staged; both give the same results, also when they share
    a slice."""
    import torch
    ctx, ref, ref_words, queries, kmers = setup
    q = queries[:90]
    pinned = torch.empty(q.size, dtype=torch.int64).pin_memory()
    pinned.numpy().view(np.uint64)[:] = q.reshape(-1)
    qp = pinned.numpy().view(np.uint64).reshape(q.shape)
    server = capi.Server(ctx, ref, slots=1, slice_queries=256, kNN=5, keep_rows=True)
    try:
        busy = server.submit(queries[200:456])       # occupies the one slot
        ts = [server.submit(qp[:40]), server.submit(q[40:90]), server.submit(qp[40:90])]
        server.wait(busy)
        server.result(busy)
        got = []
        for t in ts:
            server.wait(t)
            got.append(server.result(t)[:3])
        assert server.info()["slices_shared"] >= 1
        for a, b in zip(got[1], got[2]):
            np.testing.assert_array_equal(a, b)
        check(got[0], oracle_expected(ref_words, q[:40], kmers, 5))
    finally:
        server.close()


def test_long_knn_lists(setup):
    """kNN above the per-lane list length (radix select per row) through the
    server equals query_knn on the same queries."""
    ctx, ref, ref_words, queries, kmers = setup
    q = queries[:70]
    server = capi.Server(ctx, ref, slots=2, slice_queries=64, kNN=1000, keep_rows=True)
    try:
        t = server.submit(q)
        server.wait(t)
        idx, dist, rows, _ = server.result(t)
    finally:
        server.close()
    qry = capi.Database(ctx, q, kmers, S64)
    r, d = capi.query_knn(ctx, ref, qry, 1000, dist_col=0)
    qry.close()
    np.testing.assert_array_equal(idx, r)
    np.testing.assert_array_equal(dist, d)
    check((idx, dist, rows), oracle_expected(ref_words, q, kmers, 1000))
