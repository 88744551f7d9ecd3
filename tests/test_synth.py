"""Host-side logic of the synthetic generators (CPU only)."""
import numpy as np

from sketchlib_b200 import capi, synth

import oracle


def test_tree_shapes():
    p, t = synth.random_tree(500, seed=3)
    assert p[0] == -1 and np.all(p[1:] < np.arange(1, 500)) and np.all(p[1:] >= 0)
    assert t.shape == (500, 8) and t.dtype == np.uint32
    # resampling probability grows with k along every branch
    assert np.all(np.diff(t.astype(np.int64), axis=1) >= 0)
    p2, t2 = synth.clade_tree(1000, n_clades=20, seed=4)
    assert p2[0] == -1 and np.all(p2[1:] < np.arange(1, 1000))
    founders = np.where(p2 == 0)[0]
    assert len(founders) == 20
    pq, tq, qi = synth.query_population(p2, t2, 100, novel_frac=0.2, seed=5)
    assert len(qi) == 100 and np.all(pq[1:] < np.arange(1, len(pq)))
    assert tq.shape == (len(pq), 8)


def test_synth_host_deterministic_and_related():
    p, t = synth.random_tree(8, seed=9)
    w1 = capi.synth_host(p, t, 16, seed=123, threads=3)
    w2 = capi.synth_host(p, t, 16, seed=123, threads=1)
    np.testing.assert_array_equal(w1, w2)
    w3 = capi.synth_host(p, t, 16, seed=124, threads=2)
    assert not np.array_equal(w1, w3)
    # children share bins with their parents: far more than chance 2^-14
    for s in range(1, 8):
        c = oracle.intersize(w1[s, 0], w1[p[s], 0], 16)
        assert c > 64 * 16 * 0.3
    # and the shared fraction falls with k (longer k-mers diverge more)
    s = 5
    shares = [oracle.intersize(w1[s, k], w1[p[s], k], 16) for k in range(8)]
    assert shares[0] >= shares[-1]


def test_oracle_generator_matches_library():
    """The reference arm of the benchmark builds its inputs with the oracle's
    restatement of the generator; it must give the library's words bit for bit."""
    for n, K, s64, seed in ((40, 8, 16, 11), (300, 3, 5, 0x5EED0002), (1, 2, 4, 7)):
        kmers = list(range(15, 15 + 2 * K, 2))
        p, t = synth.random_tree(n, kmers=kmers, seed=seed)
        np.testing.assert_array_equal(oracle.synth_words(p, t, s64, seed, threads=3),
                                      capi.synth_host(p, t, s64, seed=seed, threads=2))
    p, t = synth.clade_tree(500, n_clades=7, seed=5)
    np.testing.assert_array_equal(oracle.synth_words(p, t, 8, 99),
                                  capi.synth_host(p, t, 8, seed=99))
