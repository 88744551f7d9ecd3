"""The oracle's one-pass loop (every float output of query_db for any row
range) against its single-output loops (CPU only)."""
import numpy as np

import oracle


def test_dists_multi_matches_single_output_loops():
    """The one-pass oracle (every float output, any row range) gives what the
    single-output loops give."""
    from conftest import random_sketches
    words, kmers = random_sketches(60, 5, 16, seed=4)
    rng = np.random.default_rng(2)
    table = rng.uniform(0, 0.02, (5, 2, 2)).astype(np.float32)
    cl = rng.integers(0, 2, 60).astype(np.uint16)
    spec = oracle.RandomSpec(2, True, table=table, cl_rows=cl, cl_cols=cl)
    jac, f64, f32 = oracle.dists_multi(words, kmers, 16, random=spec)
    np.testing.assert_array_equal(jac, oracle.dists(words, kmers, 16, random=spec, out_mode=1))
    np.testing.assert_array_equal(f64, oracle.dists(words, kmers, 16, random=spec, regress=0))
    np.testing.assert_array_equal(f32, oracle.dists(words, kmers, 16, random=spec, regress=1))
    j2, a2, b2 = oracle.dists_multi(words, kmers, 16, random=spec, row_begin=7, row_end=19)
    lo = 60 * 7 - 7 * 8 // 2
    hi = 60 * 19 - 19 * 20 // 2
    np.testing.assert_array_equal(j2, jac[lo:hi])
    np.testing.assert_array_equal(b2, f32[lo:hi])
    q = words[:9]
    jq, fq, _ = oracle.dists_multi(words[9:], kmers, 16, query_words=q, row_begin=3, row_end=6)
    full = oracle.dists(words[9:], kmers, 16, query_words=q, regress=0)
    np.testing.assert_array_equal(fq, full[3 * 51:6 * 51])
