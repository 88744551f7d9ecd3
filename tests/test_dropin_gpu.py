"""The drop-in pp_sketchlib module end to end on the GPU: sketch databases on
disk in the reference's layout, the reference's call signatures, results
checked against the oracle.  Mirrors the reference's own checks:
test/gpu_test.py (small_mass / small_mass_plus1 self and query distances),
test/test-dists.py:205-238 (kNN against an argsort of the square matrix,
threshold sparsification against a scan) and test/test-matrix.py (long/square
conversions)."""
import numpy as np
import pytest

import h5write
import oracle
from conftest import GOLDEN, random_sketches

pytestmark = pytest.mark.gpu
pp_sketchlib = pytest.importorskip("pp_sketchlib")

TOL = 1e-6


@pytest.fixture(scope="module")
def small_mass(tmp_path_factory):
    fx = np.load(GOLDEN / "small_mass_sketches.npz")
    d = tmp_path_factory.mktemp("small_mass")
    names = [str(n) for n in fx["names"]]
    kmers = [int(k) for k in fx["kmers"]]
    n_small = int(fx["n_small"])
    h5write.write_sketch_db(str(d / "small_mass.h5"), names[:n_small], fx["words"][:n_small],
                            kmers, 156)
    h5write.write_sketch_db(str(d / "small_mass_plus1.h5"), names, fx["words"], kmers, 156)
    return dict(ref=str(d / "small_mass"), query=str(d / "small_mass_plus1"), names=names,
                kmers=kmers, words=fx["words"], n_small=n_small, lengths=fx["length"])


def _equal_base(lengths_rows, lengths_cols):
    return oracle.RandomSpec(1, True, len_rows=lengths_rows, len_cols=lengths_cols)


def test_self_distances_small_mass(small_mass):
    s = small_mass
    r = s["names"][:s["n_small"]]
    got = pp_sketchlib.queryDatabase(s["ref"], s["ref"], r, r, s["kmers"], use_gpu=True)
    w = s["words"][:s["n_small"]]
    L = s["lengths"][:s["n_small"]]
    want = oracle.dists(w, s["kmers"], 156, random=_equal_base(L, L))
    assert got.shape == (15, 2) and got.dtype == np.float32
    np.testing.assert_allclose(got, want, atol=TOL, rtol=0)
    assert np.all(got[:, 0] > 0) and np.all(got[:, 1] > 0)   # real, related genomes


def test_query_distances_small_mass(small_mass):
    s = small_mass
    r = s["names"][:s["n_small"]]
    q = s["names"]
    got = pp_sketchlib.queryDatabase(s["ref"], s["query"], r, q, s["kmers"])
    wr, wq = s["words"][:s["n_small"]], s["words"]
    want = oracle.dists(wr, s["kmers"], 156, query_words=wq,
                        random=_equal_base(s["lengths"], s["lengths"][:s["n_small"]]))
    assert got.shape == (7 * 6, 2)
    np.testing.assert_allclose(got, want, atol=TOL, rtol=0)
    # a query identical to a reference is at distance zero
    assert np.all(got[0 * 6 + 0] == 0.0)


def test_jaccard_and_raw(small_mass):
    s = small_mass
    r = s["names"][:s["n_small"]]
    w = s["words"][:s["n_small"]]
    L = s["lengths"][:s["n_small"]]
    jac = pp_sketchlib.queryDatabase(s["ref"], s["ref"], r, r, s["kmers"], jaccard=True)
    np.testing.assert_array_equal(jac, oracle.dists(w, s["kmers"], 156, random=_equal_base(L, L),
                                                    out_mode=1))
    raw = pp_sketchlib.queryDatabase(s["ref"], s["ref"], r, r, s["kmers"], jaccard=True,
                                     random_correct=False)
    np.testing.assert_array_equal(raw, oracle.dists(w, s["kmers"], 156, out_mode=1))
    # single k-mer Jaccard, as `sketchlib query jaccard --kmer`
    one = pp_sketchlib.queryDatabase(s["ref"], s["ref"], r, r, [20], jaccard=True)
    np.testing.assert_array_equal(one[:, 0], oracle.dists(w[:, 2:3], [20], 156,
                                                          random=_equal_base(L, L),
                                                          out_mode=1)[:, 0])
    jd = pp_sketchlib.jaccardDist(s["ref"], r[0], r[1], 17, random_correct=False)
    c = oracle.intersize(w[0, 1], w[1, 1], 156)
    assert jd == oracle.jaccard(c, 156, 0.0)


def test_monte_carlo_random_table(tmp_path):
    n, nq, K = 80, 20, 8
    words, kmers = random_sketches(n + nq, K, 156, seed=91)
    kmers = np.arange(9, 9 + 2 * K, 2, dtype=np.int32)       # short k: large corrections
    names = [f"g{i:03d}" for i in range(n + nq)]
    rng = np.random.default_rng(5)
    C = 3
    bases = rng.dirichlet(np.ones(4) * 20, n + nq)
    centroids = rng.dirichlet(np.ones(4) * 20, C).astype(np.float32)
    table_names = names[: n - 10]                             # 10 references missing from it
    rand = dict(k_min=3, k_max=int(kmers[-2]) + 1, use_rc=1,  # last k >= k_max: r = 0
                table={nm: int(rng.integers(C)) for nm in table_names},
                matches={k: rng.uniform(0, 0.02, (C, C)).astype(np.float32) for k in range(3, 40)},
                centroids=centroids)
    h5write.write_sketch_db(str(tmp_path / "r.h5"), names[:n], words[:n], kmers, 156,
                            base_freq=bases[:n], random=rand)
    h5write.write_sketch_db(str(tmp_path / "q.h5"), names[n:], words[n:], kmers, 156,
                            base_freq=bases[n:])

    def closest(b):
        b = b.copy()
        b[0] = b[3] = 0.5 * (b[0] + b[3])
        b[1] = b[2] = 0.5 * (b[1] + b[2])
        return int(np.argmin(((centroids - b.astype(np.float32)) ** 2).sum(axis=1)))

    cl_ref = np.array([rand["table"].get(nm, closest(bases[i])) for i, nm in enumerate(names[:n])],
                      np.uint16)
    cl_q = np.array([closest(bases[n + i]) for i in range(nq)], np.uint16)
    table = np.zeros((K, C, C), np.float32)
    for ki, k in enumerate(kmers):
        if k < rand["k_max"]:
            table[ki] = rand["matches"][int(k)]
    r = names[:n]
    got = pp_sketchlib.queryDatabase(str(tmp_path / "r"), str(tmp_path / "r"), r, r, list(kmers),
                                     jaccard=True)
    want = oracle.dists(words[:n], kmers, 156, random=oracle.RandomSpec(
        2, True, table=table, cl_rows=cl_ref, cl_cols=cl_ref), out_mode=1)
    np.testing.assert_array_equal(got, want)
    gq = pp_sketchlib.queryDatabase(str(tmp_path / "r"), str(tmp_path / "q"), r, names[n:],
                                    list(kmers))
    wq = oracle.dists(words[:n], kmers, 156, query_words=words[n:], random=oracle.RandomSpec(
        2, True, table=table, cl_rows=cl_q, cl_cols=cl_ref))
    np.testing.assert_allclose(gq, wq, atol=TOL, rtol=0)


def test_sparse_knn_and_threshold(tmp_path):
    n = 150
    words, kmers = random_sketches(n, 8, 156, seed=17)
    names = [f"s{i:03d}" for i in range(n)]
    h5write.write_sketch_db(str(tmp_path / "db.h5"), names, words, kmers, 156)
    db = str(tmp_path / "db")
    dense = pp_sketchlib.queryDatabase(db, db, names, names, list(kmers))
    square = pp_sketchlib.longToSquare(distVec=dense[:, [0]])
    kNN = 3
    i, j, d = pp_sketchlib.querySelfSparse(ref_db_name=db, rList=names, klist=list(kmers), kNN=kNN)
    assert isinstance(i, list) and len(i) == n * kNN
    sq = square.copy()
    np.fill_diagonal(sq, np.inf)
    order = np.argsort(sq, axis=1, kind="stable")[:, :kNN]
    assert i == [r for r in range(n) for _ in range(kNN)]
    assert j == order.ravel().tolist()
    np.testing.assert_allclose(d, np.take_along_axis(sq, order, axis=1).ravel(), atol=0, rtol=0)
    cutoff = float(np.quantile(dense[:, 0], 0.1))
    ti, tj, td = pp_sketchlib.querySelfSparse(ref_db_name=db, rList=names, klist=list(kmers),
                                              dist_cutoff=cutoff)
    ei, ej = np.nonzero(np.triu(square < cutoff, k=1))
    assert ti == ei.tolist() and tj == ej.tolist()
    np.testing.assert_array_equal(np.asarray(td, np.float32), square[ei, ej])
    # accessory column and Jaccard kNN
    ai, aj, ad = pp_sketchlib.querySelfSparse(db, names, list(kmers), kNN=2, dist_col=1)
    sqa = pp_sketchlib.longToSquare(distVec=dense[:, [1]])
    np.fill_diagonal(sqa, np.inf)
    assert aj == np.argsort(sqa, axis=1, kind="stable")[:, :2].ravel().tolist()
    ji, jj, jd = pp_sketchlib.querySelfSparse(db, names, list(kmers), jaccard=True, kNN=2,
                                              dist_col=1)
    jac = pp_sketchlib.queryDatabase(db, db, names, names, list(kmers), jaccard=True)
    sqj = 1.0 - pp_sketchlib.longToSquare(distVec=jac[:, [1]])
    np.fill_diagonal(sqj, np.inf)
    assert jj == np.argsort(sqj, axis=1, kind="stable")[:, :2].ravel().tolist()


def test_matrix_transforms():
    rr = np.array([0.1, 0.2, 0.3, 0.4, 0.5, 0.6], dtype=np.float32)    # 4 references
    qq = np.array([0.8], dtype=np.float32)                             # 2 queries
    qr = np.arange(10, 18, dtype=np.float32) / 10                      # ref index fastest
    sq1 = pp_sketchlib.longToSquare(distVec=rr, num_threads=2)
    np.testing.assert_array_equal(sq1, oracle.long_to_square(rr, 4))
    assert sq1[0, 1] == rr[0] and sq1[2, 3] == rr[5] and sq1[3, 2] == rr[5]
    sq2 = pp_sketchlib.longToSquareMulti(distVec=rr, query_ref_distVec=qr,
                                         query_query_distVec=qq)
    np.testing.assert_array_equal(sq2, oracle.long_to_square(rr, 4, qr, qq, 2))
    assert sq2[1, 4] == qr[1] and sq2[0, 5] == qr[4] and sq2[4, 5] == qq[0]
    np.testing.assert_array_equal(pp_sketchlib.squareToLong(distMat=sq1, num_threads=2), rr)
    i, j, d = pp_sketchlib.sparsifyDistsByThreshold(sq2, 0.45)
    oi, oj, od = oracle.sparsify(oracle.square_to_long(sq2), 6, 0, 0.45)
    assert i == oi.tolist() and j == oj.tolist()
    np.testing.assert_array_equal(np.asarray(d, np.float32), od)


def test_api_errors(small_mass):
    s = small_mass
    r = s["names"][:s["n_small"]]
    with pytest.raises(RuntimeError, match="empty ref or query"):
        pp_sketchlib.queryDatabase(s["ref"], s["ref"], [], [], s["kmers"])
    with pytest.raises(RuntimeError, match="do not match those requested"):
        pp_sketchlib.queryDatabase(s["ref"], s["ref"], r, r, [15, 21])
    with pytest.raises(RuntimeError, match="deprecated"):
        pp_sketchlib.sparsifyDists(np.zeros((3, 3), np.float32))
    with pytest.raises(RuntimeError, match="Could not open"):
        pp_sketchlib.constructDatabase("x", ["a"], [["missing_file.fa"]], [15], 156)
    with pytest.raises(NotImplementedError):
        pp_sketchlib.addRandom("x", ["a"], [15])
    with pytest.raises(RuntimeError, match="dist_col out of range"):
        pp_sketchlib.querySelfSparse(s["ref"], r, s["kmers"], kNN=2, dist_col=3)


@pytest.mark.skipif(not oracle.ref_gpu_available(), reason="oracle/_ref/libref_gpu.so not built")
def test_semantics_gpu_matches_reference_kernel(tmp_path):
    """queryDatabase(..., semantics="gpu") reproduces the reference GPU path:
    the Monte Carlo table is copied up to k_max inclusive (flattened_random,
    src/random/random_match.cpp:300) and indexed [k][ref cluster][query
    cluster], and the fit is the reference kernel's, bit for bit."""
    n, nq, K = 80, 20, 6
    words, _ = random_sketches(n + nq, K, 64, seed=93)
    kmers = np.arange(11, 11 + 2 * K, 2, dtype=np.int32)
    names = [f"s{i:03d}" for i in range(n + nq)]
    rng = np.random.default_rng(9)
    C = 3
    centroids = rng.dirichlet(np.ones(4) * 20, C).astype(np.float32)
    bases = rng.dirichlet(np.ones(4) * 20, n + nq)
    rand = dict(k_min=3, k_max=int(kmers[-1]), use_rc=1,        # last k == k_max: GPU keeps it
                table={nm: int(rng.integers(C)) for nm in names[:n]},
                matches={k: rng.uniform(0, 0.02, (C, C)).astype(np.float32) for k in range(3, 40)},
                centroids=centroids)
    h5write.write_sketch_db(str(tmp_path / "r.h5"), names[:n], words[:n], kmers, 64,
                            base_freq=bases[:n], random=rand)
    h5write.write_sketch_db(str(tmp_path / "q.h5"), names[n:], words[n:], kmers, 64,
                            base_freq=bases[n:])
    info = pp_sketchlib._load_random(str(tmp_path / "r"))
    table = np.stack([rand["matches"][int(k)] for k in kmers]).astype(np.float32)
    cl_ref = np.array([rand["table"][nm] for nm in names[:n]], np.uint16)
    r = names[:n]
    got = pp_sketchlib.queryDatabase(str(tmp_path / "r"), str(tmp_path / "r"), r, r, list(kmers),
                                     use_gpu=True, semantics="gpu")
    want = oracle.RefGpuKernel().dists(words[:n], kmers, 64, table=table, ref_lookup=cl_ref)
    np.testing.assert_array_equal(got, want)
    # the default follows the CPU path, which differs
    cpu = pp_sketchlib.queryDatabase(str(tmp_path / "r"), str(tmp_path / "r"), r, r, list(kmers))
    assert np.any(cpu != want)
    assert info["k_max"] == int(kmers[-1])
    with pytest.raises(ValueError):
        pp_sketchlib.queryDatabase(str(tmp_path / "r"), str(tmp_path / "r"), r, r, list(kmers),
                                   semantics="fast")


def test_many_samples_read_while_computing(tmp_path):
    """Databases of several upload chunks: the words are read on background
    threads while the call runs (all-vs-all from the last samples down, query
    mode queries first), the rows return through the page-locked stage; the
    result equals the oracle's, in the caller's sample order, and a repeat
    call (reused stages) gives the same array."""
    n, nq, K, s64 = 1300, 150, 4, 16
    words, kmers = random_sketches(n + nq, K, s64, seed=95)
    names = [f"s{i:05d}" for i in range(n + nq)]
    rng = np.random.default_rng(9)
    lengths = rng.integers(1_000_000, 5_000_000, n + nq)
    h5write.write_sketch_db(str(tmp_path / "r.h5"), names[:n], words[:n], kmers, s64,
                            lengths=lengths[:n])
    h5write.write_sketch_db(str(tmp_path / "q.h5"), names[n:], words[n:], kmers, s64,
                            lengths=lengths[n:])
    order = list(rng.permutation(n))                  # not the file's order
    r = [names[i] for i in order]
    got = pp_sketchlib.queryDatabase(str(tmp_path / "r"), str(tmp_path / "r"), r, r, list(kmers))
    L = lengths[order].astype(np.uint64)
    want = oracle.dists(words[order], kmers, s64, random=_equal_base(L, L))
    np.testing.assert_allclose(got, want, atol=TOL, rtol=0)
    again = pp_sketchlib.queryDatabase(str(tmp_path / "r"), str(tmp_path / "r"), r, r, list(kmers))
    np.testing.assert_array_equal(again, got)
    q = names[n:]
    gq = pp_sketchlib.queryDatabase(str(tmp_path / "r"), str(tmp_path / "q"), r, q, list(kmers),
                                    random_correct=False)
    wq = oracle.dists(words[order], kmers, s64, query_words=words[n:])
    np.testing.assert_allclose(gq, wq, atol=TOL, rtol=0)
    with pytest.raises(pp_sketchlib.HDF5Exception, match="Missing sketch"):
        pp_sketchlib.queryDatabase(str(tmp_path / "r"), str(tmp_path / "r"), r + ["nope"],
                                   r + ["nope"], list(kmers))
