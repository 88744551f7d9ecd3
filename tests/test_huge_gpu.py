"""An all-vs-all past 2^31 pairs: 66,000 samples, K = 8, sketchsize64 156 ->
2,177,967,000 pairs (17.4 GB of core/accessory in HBM).  The reference's GPU
kernel indexes pairs with 32-bit ints (src/gpu/dist.cu:174); here every index
is 64-bit.  The pairs among the last 1,500 samples, whose long-form rows all
lie above 2^31, are checked against the oracle; the same samples as queries
against all 66,000 references give those pairs bit-identically."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

N = 66_000
KMERS = list(range(15, 31, 2))
S64 = 156
TAIL = 1_500
SEED = 0x5EED0066


def test_all_vs_all_beyond_two_to_the_31_pairs(gpu_ctx):
    import torch
    from sketchlib_b200 import capi, synth
    assert N * (N - 1) // 2 > 2 ** 31
    wps = len(KMERS) * S64 * 14
    parent, thresh = synth.clade_tree(N, n_clades=200, kmers=KMERS, seed=SEED)
    words = torch.empty(N * wps, dtype=torch.int64, device="cuda")
    capi.synth_device(gpu_ctx, parent, thresh, S64, seed=SEED, d_words=words.data_ptr())
    db = capi.Database(gpu_ctx, words.data_ptr(), KMERS, S64, n_samples=N)
    tail = words.view(N, wps)[N - TAIL:].cpu().numpy().view(np.uint64).reshape(TAIL, len(KMERS), -1)
    del words
    out = torch.empty((N * (N - 1) // 2, 2), dtype=torch.float32, device="cuda")
    capi.dists_dense(gpu_ctx, db, out=out.data_ptr())
    gpu_ctx.synchronize()
    # condensed rows of the pairs (i, j), N - TAIL <= i < j < N
    i, j = np.triu_indices(TAIL, 1)
    gi = torch.as_tensor(i + N - TAIL, device="cuda")
    gj = torch.as_tensor(j + N - TAIL, device="cuda")
    rows = gi * (2 * N - gi - 1) // 2 + (gj - gi - 1)
    assert int(rows.min()) > 2 ** 31
    got = out[rows].cpu().numpy()
    del out
    want = oracle.dists(tail, KMERS, S64)
    np.testing.assert_allclose(got, want, atol=1e-6, rtol=0)
    # the tail as queries against every reference: row q, column N - TAIL + j
    qdb = capi.Database(gpu_ctx, tail, KMERS, S64)
    qout = torch.empty((TAIL * N, 2), dtype=torch.float32, device="cuda")
    capi.dists_dense(gpu_ctx, db, qdb, out=qout.data_ptr())
    gpu_ctx.synchronize()
    qrows = torch.as_tensor(i * N + (N - TAIL) + j, device="cuda")
    np.testing.assert_array_equal(qout[qrows].cpu().numpy(), got)
    db.close()
    qdb.close()
