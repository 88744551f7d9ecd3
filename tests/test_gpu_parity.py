"""GPU parity: the CUDA path through the C ABI against the CPU oracle.

Bars: intersection counts and Jaccard floats bit-exact; core/accessory within
1e-6 of the oracle's double-precision fit (the same arithmetic in the same
order) and within 1e-5 of the float LDLT restatement of the reference's
fit_slope wherever that float solve is well conditioned (tests/fp_error.py);
kNN / threshold / long-square outputs exact.
"""
import numpy as np
import pytest

import oracle
from conftest import random_sketches
from sketchlib_b200 import capi

pytestmark = pytest.mark.gpu

import fp_error

TOL_F64 = fp_error.TOL_F64   # GPU vs oracle, both double-precision fits

SHAPES = [  # (n, K, s64)
    (1, 2, 16), (2, 2, 16), (31, 3, 1), (33, 8, 156), (65, 8, 156), (130, 4, 64),
    (257, 8, 16), (70, 14, 16), (40, 16, 2), (50, 1, 156), (96, 8, 312),
]


def _db(ctx, words, kmers, s64, **kw):
    return capi.Database(ctx, words, kmers, s64, **kw)


@pytest.mark.parametrize("n,K,s64", SHAPES)
def test_counts_bit_exact_self(gpu_ctx, n, K, s64):
    words, kmers = random_sketches(n, K, s64, seed=1000 + n * 7 + K)
    db = _db(gpu_ctx, words, kmers, s64)
    got = capi.dists_dense(gpu_ctx, db, out_mode=capi.OUT_COUNTS)
    want = oracle.dists(words, kmers, s64, out_mode=2)
    assert got.shape == want.shape
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("nq,nr,K,s64", [(1, 1, 2, 16), (5, 300, 8, 156), (129, 64, 3, 16),
                                         (70, 200, 14, 16), (64, 64, 8, 1)])
def test_counts_bit_exact_query(gpu_ctx, nq, nr, K, s64):
    rw, kmers = random_sketches(nr, K, s64, seed=77 + nr)
    qw, _ = random_sketches(nq, K, s64, seed=99 + nq)
    ref = _db(gpu_ctx, rw, kmers, s64)
    qry = _db(gpu_ctx, qw, kmers, s64)
    got = capi.dists_dense(gpu_ctx, ref, qry, out_mode=capi.OUT_COUNTS)
    want = oracle.dists(rw, kmers, s64, query_words=qw, out_mode=2)
    np.testing.assert_array_equal(got, want)


def test_unrelated_and_identical_sketches(gpu_ctx):
    words, kmers = random_sketches(40, 8, 156, seed=5, related=False)
    words[7] = words[3]                  # an identical pair: every bin matches
    db = _db(gpu_ctx, words, kmers, 156)
    got = capi.dists_dense(gpu_ctx, db, out_mode=capi.OUT_COUNTS)
    np.testing.assert_array_equal(got, oracle.dists(words, kmers, 156, out_mode=2))
    pos = 40 * 3 - 3 * 4 // 2 + 7 - 1 - 3
    assert np.all(got[pos] == 64 * 156)
    ca = capi.dists_dense(gpu_ctx, db)
    assert np.all(ca[pos] == 0.0)


def _random_variants(n_rows, n_cols, K, self_, seed):
    rng = np.random.default_rng(seed)
    C = 3
    table = rng.uniform(0, 0.01, size=(K, C, C)).astype(np.float32)
    cl_r = rng.integers(0, C, n_rows).astype(np.uint16)
    cl_c = cl_r if self_ else rng.integers(0, C, n_cols).astype(np.uint16)
    len_r = rng.integers(1_500_000, 6_000_000, n_rows).astype(np.uint64)
    len_c = len_r if self_ else rng.integers(1_500_000, 6_000_000, n_cols).astype(np.uint64)
    return table, (cl_r, cl_c), (len_r, len_c)


@pytest.mark.parametrize("mode", ["none", "equal_base", "table"])
@pytest.mark.parametrize("self_", [True, False])
def test_jaccard_and_coreacc(gpu_ctx, mode, self_):
    K, s64 = 8, 156
    nr, nq = 150, 70
    rw, kmers = random_sketches(nr, K, s64, seed=21)
    kmers = np.arange(11, 11 + 2 * K, 2, dtype=np.int32)   # short k: real correction
    qw = None if self_ else random_sketches(nq, K, s64, seed=22)[0]
    table, (cl_q, cl_r), (len_q, len_r) = _random_variants(nr if self_ else nq, nr, K, self_, 3)
    ref = _db(gpu_ctx, rw, kmers, s64, cluster=cl_r, seq_len=len_r)
    qry = None if self_ else _db(gpu_ctx, qw, kmers, s64, cluster=cl_q, seq_len=len_q)
    if mode == "none":
        rnd, spec = None, oracle.RandomSpec()
    elif mode == "equal_base":
        rnd = capi.Random(gpu_ctx, capi.RANDOM_EQUAL_BASE, kmers, use_rc=True)
        spec = oracle.RandomSpec(1, True, len_rows=len_q, len_cols=len_r)
    else:
        rnd = capi.Random(gpu_ctx, capi.RANDOM_TABLE, kmers, table=table)
        spec = oracle.RandomSpec(2, True, table=table, cl_rows=cl_q, cl_cols=cl_r)
    jac = capi.dists_dense(gpu_ctx, ref, qry, rnd, out_mode=capi.OUT_JACCARD)
    want_j = oracle.dists(rw, kmers, s64, query_words=qw, random=spec, out_mode=1)
    np.testing.assert_array_equal(jac, want_j)
    if mode != "none":
        raw = oracle.dists(rw, kmers, s64, query_words=qw, out_mode=1)
        assert np.any(raw != want_j)             # the correction changed something
    ca = capi.dists_dense(gpu_ctx, ref, qry, rnd)
    want64 = oracle.dists(rw, kmers, s64, query_words=qw, random=spec, regress=0)
    want32 = oracle.dists(rw, kmers, s64, query_words=qw, random=spec, regress=1)
    # exact fit bar on every pair; the 1e-5 bar against the reference's float
    # arithmetic on the pairs where that arithmetic is well conditioned
    fp_error.check(jac, want_j, ca, want64, want32)
    assert np.mean(ca == want64) > 0.99


def test_cluster_ids_beyond_the_random_table_are_refused(gpu_ctx):
    """A cluster id >= the table's cluster count would index past the table
    (and its count tables) on the device: refused before any launch."""
    K, s64 = 4, 16
    words, kmers = random_sketches(100, K, s64, seed=23)
    table = np.full((K, 3, 3), 0.001, np.float32)
    rnd = capi.Random(gpu_ctx, capi.RANDOM_TABLE, kmers, table=table)
    ok = _db(gpu_ctx, words, kmers, s64, cluster=np.full(100, 2, np.uint16))
    capi.dists_dense(gpu_ctx, ok, None, rnd)
    bad = _db(gpu_ctx, words, kmers, s64, cluster=np.r_[np.zeros(99), 3].astype(np.uint16))
    with pytest.raises(capi.SketchlibError, match="beyond the 3 clusters"):
        capi.dists_dense(gpu_ctx, bad, None, rnd)
    with pytest.raises(capi.SketchlibError, match="beyond the 3 clusters"):
        capi.dists_dense(gpu_ctx, ok, bad, rnd)


@pytest.mark.parametrize("cfg", [c["id"] for c in capi.tile_configs()])
def test_every_tile_shape_agrees(gpu_ctx, cfg):
    info = {c["id"]: c for c in capi.tile_configs()}[cfg]
    K = min(4, info["max_kmers"])
    words, kmers = random_sketches(300, K, 16, seed=40 + cfg)
    db = _db(gpu_ctx, words, kmers, 16)
    gpu_ctx.set_tile_config(cfg)
    try:
        got = capi.dists_dense(gpu_ctx, db, out_mode=capi.OUT_COUNTS)
        qw, _ = random_sketches(77, K, 16, seed=50 + cfg)
        q = _db(gpu_ctx, qw, kmers, 16)
        gotq = capi.dists_dense(gpu_ctx, db, q, out_mode=capi.OUT_COUNTS)
    finally:
        gpu_ctx.set_tile_config(0)
    np.testing.assert_array_equal(got, oracle.dists(words, kmers, 16, out_mode=2))
    np.testing.assert_array_equal(gotq, oracle.dists(words, kmers, 16, query_words=qw, out_mode=2))


@pytest.mark.parametrize("cfg", [1, 4])
def test_counts_at_the_maximum_sketch_width(gpu_ctx, cfg):
    """sketchsize64 1023: identical samples count 64 * 1023 = 65,472 bins per
    k, the most a 16-bit count holds; two counts share a register in the
    kernel, so a carry out of the low half would corrupt the neighbour."""
    s64, K = 1023, 2
    words, kmers = random_sketches(40, K, s64, seed=77, related=False)
    words[1::3] = words[0]                      # many identical pairs
    words[2, :, :] = ~words[0]                  # all planes differ from sample 0
    db = _db(gpu_ctx, words, kmers, s64)
    gpu_ctx.set_tile_config(cfg)
    try:
        got = capi.dists_dense(gpu_ctx, db, out_mode=capi.OUT_COUNTS)
    finally:
        gpu_ctx.set_tile_config(0)
    want = oracle.dists(words, kmers, s64, out_mode=2)
    assert want.max() == 64 * s64
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("s64,cfg", [(1024, 1), (1562, 1), (2047, 4), (3070, 6), (4100, 1)])
def test_counts_beyond_one_counter(gpu_ctx, s64, cfg):
    """Sketches wider than one 16-bit counter (64 * s64 > 65,535 bins per k)
    are counted in chunks of 2,046 blocks, each in its own count slot, and
    summed: identical samples count every bin, complementary ones none."""
    K = 2
    words, kmers = random_sketches(20, K, s64, seed=s64, related=False)
    words[1::3] = words[0]
    words[2, :, :] = ~words[0]
    db = _db(gpu_ctx, words, kmers, s64)
    gpu_ctx.set_tile_config(cfg)
    try:
        got = capi.dists_dense(gpu_ctx, db, out_mode=capi.OUT_COUNTS)
        qdb = _db(gpu_ctx, words[:7], kmers, s64)
        gotq = capi.dists_dense(gpu_ctx, db, qdb, out_mode=capi.OUT_COUNTS)
    finally:
        gpu_ctx.set_tile_config(0)
    want = oracle.dists(words, kmers, s64, out_mode=2)
    assert want.max() == 64 * s64
    np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(gotq, oracle.dists(words, kmers, s64, query_words=words[:7],
                                                     out_mode=2))


@pytest.mark.parametrize("case", ["wide", "many_k"])
def test_reference_scale_parameters(gpu_ctx, case):
    """Parameters the reference accepts and this build once refused: sketch
    size 100,000 (sketchsize64 1562, pp_sketch/__main__.py:138) and the k set
    13..101 step 2 (K = 45).  Self and query, every output mode, the
    host-in call and a batch: counts and Jaccards exact, core/accessory within
    the double-fit bar of the oracle."""
    import torch
    from sketchlib_b200 import synth
    if case == "wide":
        kmers, s64, n = np.arange(15, 23, 2, dtype=np.int32), 1562, 160
    else:
        kmers, s64, n = np.arange(13, 102, 2, dtype=np.int32), 16, 300
    parent, thresh = synth.random_tree(n, kmers=kmers, seed=0x5EED0045, c_max=0.01, a_max=0.1)
    words = capi.synth_host(parent, thresh, s64, seed=0x5EED0045)
    qw = words[:50]
    ref = _db(gpu_ctx, words, kmers, s64)
    qry = _db(gpu_ctx, qw, kmers, s64)
    for q, qwords in ((None, None), (qry, qw)):
        np.testing.assert_array_equal(
            capi.dists_dense(gpu_ctx, ref, q, out_mode=capi.OUT_COUNTS),
            oracle.dists(words, kmers, s64, query_words=qwords, out_mode=2))
        np.testing.assert_array_equal(
            capi.dists_dense(gpu_ctx, ref, q, out_mode=capi.OUT_JACCARD),
            oracle.dists(words, kmers, s64, query_words=qwords, out_mode=1))
        want = oracle.dists(words, kmers, s64, query_words=qwords)
        got = capi.dists_dense(gpu_ctx, ref, q)
        assert np.abs(got - want).max() <= TOL_F64
        assert (want[:, 0] > 0).mean() > 0.5
    got = capi.query_db(gpu_ctx, words, kmers, s64)
    assert np.abs(got - oracle.dists(words, kmers, s64)).max() <= TOL_F64
    out = torch.full((capi.dists_rows(ref, qry), 2), -7.0, dtype=torch.float32, device="cuda")
    b = capi.Batch(gpu_ctx, [(ref, qry, None, capi.OUT_CORE_ACC, out.data_ptr())])
    b.run()
    b.close()
    assert np.abs(out.cpu().numpy() - oracle.dists(words, kmers, s64, query_words=qw)).max() \
        <= TOL_F64


def test_pack_roundtrip_and_synth_device(gpu_ctx):
    import torch
    from sketchlib_b200 import synth
    p, t = synth.random_tree(300, seed=8)
    host = capi.synth_host(p, t, 156, seed=31)
    dev = torch.empty(host.size, dtype=torch.int64, device="cuda")
    capi.synth_device(gpu_ctx, p, t, 156, seed=31, d_words=dev.data_ptr())
    np.testing.assert_array_equal(dev.cpu().numpy().view(np.uint64).reshape(host.shape), host)
    db = capi.Database(gpu_ctx, dev.data_ptr(), list(range(15, 31, 2)), 156, n_samples=300)
    np.testing.assert_array_equal(db.download(), host)


@pytest.mark.parametrize("jaccard,dist_col", [(False, 0), (False, 1), (True, 1)])
def test_knn_self(gpu_ctx, jaccard, dist_col):
    n, K, s64, knn = 200, 8, 156, 10
    words, kmers = random_sketches(n, K, s64, seed=61)
    words[10] = words[11]                  # ties at distance 0
    words[12] = words[11]
    db = _db(gpu_ctx, words, kmers, s64)
    i, j, d = capi.dists_knn(gpu_ctx, db, knn, dist_col=dist_col, jaccard=jaccard)
    # selection is checked on the GPU's own dense values (their parity with the
    # oracle is covered above), so near-ties cannot flip on an ulp
    if jaccard:
        dense = capi.dists_dense(gpu_ctx, db, out_mode=capi.OUT_JACCARD)
        np.testing.assert_array_equal(dense, oracle.dists(words, kmers, s64, out_mode=1))
        oi, oj, od = oracle.knn_self(dense, n, dist_col, knn, jaccard_=True)
    else:
        dense = capi.dists_dense(gpu_ctx, db)
        oi, oj, od = oracle.knn_self(dense, n, dist_col, knn)
    np.testing.assert_array_equal(i, oi)
    np.testing.assert_array_equal(j, oj)
    np.testing.assert_allclose(d, od, atol=TOL_F64, rtol=0)
    if not jaccard:
        # the reference test's check: indices equal a stable argsort of the square rows
        sq = oracle.long_to_square(dense[:, dist_col], n)
        np.fill_diagonal(sq, np.inf)
        order = np.argsort(sq, axis=1, kind="stable")[:, :knn]
        np.testing.assert_array_equal(j.reshape(n, knn), order)


def test_query_knn(gpu_ctx):
    nr, nq, K, s64, knn = 500, 37, 8, 156, 5
    rw, kmers = random_sketches(nr, K, s64, seed=71)
    qw = rw[:nq].copy()                        # queries identical to some refs
    ref = _db(gpu_ctx, rw, kmers, s64)
    qry = _db(gpu_ctx, qw, kmers, s64)
    r, d = capi.query_knn(gpu_ctx, ref, qry, knn, dist_col=0)
    dense = capi.dists_dense(gpu_ctx, ref, qry)[:, 0].reshape(nq, nr)
    order = np.argsort(dense, axis=1, kind="stable")[:, :knn]
    np.testing.assert_array_equal(r, order)
    np.testing.assert_allclose(d, np.take_along_axis(dense, order, axis=1), atol=TOL_F64, rtol=0)


@pytest.mark.parametrize("cutoff", [0.0, 0.02, 0.5, 2.0])
def test_threshold_sparse(gpu_ctx, cutoff):
    n, K, s64 = 180, 8, 156
    words, kmers = random_sketches(n, K, s64, seed=81)
    db = _db(gpu_ctx, words, kmers, s64)
    i, j, d = capi.dists_threshold(gpu_ctx, db, 0, cutoff)
    dense = capi.dists_dense(gpu_ctx, db)
    oi, oj, od = oracle.sparsify(dense, n, 0, cutoff)
    np.testing.assert_array_equal(i, oi)
    np.testing.assert_array_equal(j, oj)
    np.testing.assert_array_equal(d, od)
    # the host long-form entry point gives the same entries
    i2, j2, d2 = capi.sparse_threshold(gpu_ctx, dense, n, 0, cutoff)
    np.testing.assert_array_equal(i2, oi)
    np.testing.assert_array_equal(d2, od)


def test_long_square_roundtrip(gpu_ctx):
    rng = np.random.default_rng(4)
    n_rr, n_qq = 37, 5
    rr = rng.random(n_rr * (n_rr - 1) // 2).astype(np.float32)
    qr = rng.random(n_rr * n_qq).astype(np.float32)
    qq = rng.random(n_qq * (n_qq - 1) // 2).astype(np.float32)
    sq = capi.long_to_square(gpu_ctx, rr, qr, qq, n_qq)
    np.testing.assert_array_equal(sq, oracle.long_to_square(rr, n_rr, qr, qq, n_qq))
    sq1 = capi.long_to_square(gpu_ctx, rr)
    np.testing.assert_array_equal(capi.square_to_long(gpu_ctx, sq1), rr)
    np.testing.assert_array_equal(sq1, oracle.long_to_square(rr, n_rr))


def test_errors_and_edges(gpu_ctx):
    w, kmers = random_sketches(10, 4, 16, seed=1)
    w2, _ = random_sketches(10, 4, 32, seed=2)
    a = _db(gpu_ctx, w, kmers, 16)
    b = _db(gpu_ctx, w2, kmers, 32)
    with pytest.raises(capi.SketchlibError, match="Mismatching sketchsize64"):
        capi.dists_dense(gpu_ctx, a, b)
    c = _db(gpu_ctx, w, kmers + 2, 16)
    with pytest.raises(capi.SketchlibError, match="Mismatching k-mer lengths"):
        capi.dists_dense(gpu_ctx, a, c)
    with pytest.raises(capi.SketchlibError, match="dist_col out of range"):
        capi.dists_knn(gpu_ctx, a, 2, dist_col=2)
    with pytest.raises(capi.SketchlibError, match="at least 0"):
        capi.dists_threshold(gpu_ctx, a, 0, -1.0)
    with pytest.raises(capi.SketchlibError, match="bbits"):
        capi.Database(gpu_ctx, np.zeros((2, 4, 16 * 13), np.uint64), kmers, 16, bbits=13)
    one = _db(gpu_ctx, w[:1], kmers, 16)
    assert capi.dists_dense(gpu_ctx, one).shape == (0, 2)
    empty = capi.Database(gpu_ctx, np.zeros((0, 4, 16 * 14), np.uint64), kmers, 16)
    with pytest.raises(capi.SketchlibError, match="empty ref or query"):
        capi.dists_dense(gpu_ctx, empty)


def test_device_output_and_large_properties(gpu_ctx):
    """Full-size all-vs-all (4,096 samples, 8 k x 156 x 14): results written to
    device memory, checked exactly against the oracle on a seeded sample of
    pairs, and self-mode must equal query-mode on the same database."""
    import torch
    from sketchlib_b200 import synth
    n, s64 = 4096, 156
    kmers = list(range(15, 31, 2))
    p, t = synth.random_tree(n, kmers=kmers, seed=0x5EED0002)
    dwords = torch.empty(n * 8 * s64 * 14, dtype=torch.int64, device="cuda")
    capi.synth_device(gpu_ctx, p, t, s64, seed=0x5EED0002, d_words=dwords.data_ptr())
    db = capi.Database(gpu_ctx, dwords.data_ptr(), kmers, s64, n_samples=n)
    pairs = n * (n - 1) // 2
    out = torch.full((pairs, 2), -1.0, dtype=torch.float32, device="cuda")
    capi.dists_dense(gpu_ctx, db, out=out.data_ptr())
    gpu_ctx.synchronize()
    res = out.cpu().numpy()
    assert np.all(res >= 0) and np.all(res <= 1)
    rng = np.random.default_rng(0)
    rows = np.sort(rng.choice(n, 24, replace=False))
    host = dwords.cpu().numpy().view(np.uint64).reshape(n, 8, s64 * 14)
    sub = oracle.dists(host, kmers, s64, query_words=host[rows])   # rows vs all
    for a, i in enumerate(rows):
        j = np.arange(i + 1, n)
        pos = n * i - i * (i + 1) // 2 + j - 1 - i
        np.testing.assert_allclose(res[pos], sub[a * n + j], atol=TOL_F64, rtol=0)
    qdb = capi.Database(gpu_ctx, host[rows], kmers, s64)
    q = capi.dists_dense(gpu_ctx, db, qdb)
    np.testing.assert_allclose(q, sub, atol=TOL_F64, rtol=0)


def test_context_outlives_its_handles():
    """Destroying a context before its databases is safe: the handles keep it
    alive and the last one to go frees it."""
    ctx = capi.Context(0)
    w, kmers = random_sketches(20, 2, 16, seed=3)
    db = capi.Database(ctx, w, kmers, 16)
    rnd = capi.Random(ctx, capi.RANDOM_EQUAL_BASE, kmers)
    capi.lib.sk_ctx_destroy(ctx.handle)
    ctx.handle = None
    rnd.close()
    db.close()


@pytest.mark.parametrize("query", [False, True])
def test_maximum_kmer_count(gpu_ctx, query):
    """K = 128 (the most this build takes), k = 5..132: counts bit-exact,
    Jaccard exact, core/accessory within the double-fit bar."""
    from sketchlib_b200 import synth
    kmers = np.arange(5, 133, dtype=np.int32)
    parent, thresh = synth.random_tree(90, kmers=kmers, seed=0x5EED0032, c_max=0.01)
    words = capi.synth_host(parent, thresh, 8, seed=0x5EED0032)
    rw, qw = (words[30:], words[:30]) if query else (words, None)
    ref = _db(gpu_ctx, rw, kmers, 8)
    qry = _db(gpu_ctx, qw, kmers, 8) if query else None
    np.testing.assert_array_equal(capi.dists_dense(gpu_ctx, ref, qry, out_mode=capi.OUT_COUNTS),
                                  oracle.dists(rw, kmers, 8, query_words=qw, out_mode=2))
    np.testing.assert_array_equal(capi.dists_dense(gpu_ctx, ref, qry, out_mode=capi.OUT_JACCARD),
                                  oracle.dists(rw, kmers, 8, query_words=qw, out_mode=1))
    got = capi.dists_dense(gpu_ctx, ref, qry)
    want = oracle.dists(rw, kmers, 8, query_words=qw)
    assert np.abs(got - want).max() <= TOL_F64
    assert (want[:, 0] > 0).mean() > 0.5                  # the fits are not all degenerate
