"""The large all-vs-all at full size: 31,610 samples (200 clades with
log-normal sizes), K = 8, sketchsize64 156 -- 499,580,245 pairs in a 4.0 GB
device long form, plus the kNN = 10 graph.

The oracle cannot redo 5e8 pairs in a test, so parity is split:
* sampled rows (first, last, interior) against the oracle (1e-6, both
  double-precision fits), covering both halves of each row of the condensed
  matrix (pairs (i, r) with i < r and (r, j) with j > r);
* a size-independent property over every column of those rows: the same
  samples as a separate query database give bit-identical values through the
  query-vs-reference kernel path;
* kNN: the whole graph has the reference's shape (i repeated kNN times, j != i,
  distances ascending) and, for the sampled rows, equals the kNN = 10 smallest
  of the device's own dense row by (distance, j).
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

N = 31_610
KMERS = list(range(15, 31, 2))
S64 = 156
SEED = 0x5EED0003
ROWS = [0, 1, 4_097, 15_805, 31_608, 31_609]
KNN = 10


def condensed(i, j, n):
    """square_to_condensed (src/dist/matrix_idx.hpp:46-50) for i < j."""
    return i * (2 * n - i - 1) // 2 + (j - i - 1)


@pytest.fixture(scope="module")
def large(gpu_ctx):
    import torch
    from sketchlib_b200 import capi, synth
    parent, thresh = synth.clade_tree(N, n_clades=200, kmers=KMERS, seed=SEED)
    words = torch.empty(N * len(KMERS) * S64 * 14, dtype=torch.int64, device="cuda")
    capi.synth_device(gpu_ctx, parent, thresh, S64, seed=SEED, d_words=words.data_ptr())
    db = capi.Database(gpu_ctx, words.data_ptr(), KMERS, S64, n_samples=N)
    out = torch.empty((N * (N - 1) // 2, 2), dtype=torch.float32, device="cuda")
    capi.dists_dense(gpu_ctx, db, out=out.data_ptr())
    gpu_ctx.synchronize()
    host_words = words.cpu().numpy().view(np.uint64).reshape(N, len(KMERS), S64 * 14)
    del words
    # full rows ROWS x N (self pair included as 0) gathered from the condensed form
    r = torch.as_tensor(ROWS, device="cuda")[:, None]
    c = torch.arange(N, device="cuda")[None, :]
    lo, hi = torch.minimum(r, c), torch.maximum(r, c)
    idx = condensed(lo, hi, N).clamp(min=0)
    rows = out[idx.reshape(-1)].reshape(len(ROWS), N, 2)
    rows[(r == c).expand(-1, N)] = 0.0
    yield db, host_words, rows.cpu().numpy(), out
    db.close()


def test_large_sampled_rows_vs_oracle(large):
    db, host_words, rows, _ = large
    want = oracle.dists(host_words, KMERS, S64, query_words=host_words[ROWS])
    want = want.reshape(len(ROWS), N, 2)
    for q, r in enumerate(ROWS):
        want[q, r] = 0.0
    assert np.isfinite(rows).all()
    np.testing.assert_allclose(rows, want, atol=1e-6, rtol=0)


def test_large_rows_through_query_path_bit_identical(gpu_ctx, large):
    from sketchlib_b200 import capi
    db, host_words, rows, _ = large
    qdb = capi.Database(gpu_ctx, np.ascontiguousarray(host_words[ROWS]), KMERS, S64)
    got = capi.dists_dense(gpu_ctx, db, qdb).reshape(len(ROWS), N, 2)
    qdb.close()
    for q, r in enumerate(ROWS):
        got[q, r] = 0.0             # query mode computes the self pair; self mode has none
    np.testing.assert_array_equal(got, rows)


def test_large_knn_graph(gpu_ctx, large):
    from sketchlib_b200 import capi
    db, _, rows, out = large
    del out
    i, j, d = capi.dists_knn(gpu_ctx, db, KNN, dist_col=0)
    assert len(i) == N * KNN
    np.testing.assert_array_equal(i, np.repeat(np.arange(N), KNN))
    assert (j != i).all() and (j >= 0).all() and (j < N).all()
    dd = d.reshape(N, KNN)
    assert (np.diff(dd, axis=1) >= 0).all()
    jj = j.reshape(N, KNN)
    for q, r in enumerate(ROWS):
        row = rows[q, :, 0].astype(np.float64)
        row[r] = np.inf
        order = np.lexsort((np.arange(N), row))[:KNN]
        np.testing.assert_array_equal(jj[r], order)
        np.testing.assert_array_equal(dd[r], rows[q, order, 0])
