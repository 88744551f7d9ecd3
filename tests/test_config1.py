"""The CPU-runnable parity case: synthetic genomes sketched by the reference's
own sketcher (oracle/_ref/libref_sketch.so, built from src/sketch/*.cpp), then
distances through the CUDA path against the oracle.  Skipped where the
reference sketcher was not built."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.skipif(not oracle.sketcher_available(),
                                reason="oracle/_ref/libref_sketch.so not built")

KMERS = list(range(15, 31, 2))   # k = 15, 17, ..., 29
S64 = 156                        # sketch_size 10000
SEED = 0x5EED0001


def test_reference_sketcher_is_deterministic_and_sane():
    rs = oracle.RefSketcher()
    g = rs.genomes(6, 300_000, SEED)
    g[5] = g[2]                                  # an identical genome
    a = rs.sketch(g, KMERS, S64, threads=4)
    b = rs.sketch(g, KMERS, S64, threads=1)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(a[5], a[2])
    J = oracle.dists(a, KMERS, S64, out_mode=1)
    # Jaccard falls with k for related genomes (1.0 for the identical pair)
    assert np.all(np.diff(J, axis=1) <= 1e-3)
    ref = oracle.RefQueryDb()
    for i in range(5):
        assert oracle.intersize(a[i, 0], a[i + 1, 0], S64) == ref.intersize(a[i, 0], a[i + 1, 0], S64)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["none", "equal_base", "table"])
def test_config1_genomes_gpu_vs_oracle(gpu_ctx, mode):
    from sketchlib_b200 import capi
    rs = oracle.RefSketcher()
    genomes = rs.genomes(64, 2_500_000, SEED)
    words = rs.sketch(genomes, KMERS, S64)
    lens = np.full(64, 2_500_000, np.uint64)
    rng = np.random.default_rng(1)
    cl = rng.integers(0, 3, 64).astype(np.uint16)
    table = rng.uniform(0, 0.003, (len(KMERS), 3, 3)).astype(np.float32)   # fabricated C = 3
    db = capi.Database(gpu_ctx, words, KMERS, S64, cluster=cl, seq_len=lens)
    if mode == "none":
        rnd, spec = None, oracle.RandomSpec()
    elif mode == "equal_base":
        rnd = capi.Random(gpu_ctx, capi.RANDOM_EQUAL_BASE, KMERS)
        spec = oracle.RandomSpec(1, True, len_rows=lens, len_cols=lens)
    else:
        rnd = capi.Random(gpu_ctx, capi.RANDOM_TABLE, KMERS, table=table)
        spec = oracle.RandomSpec(2, True, table=table, cl_rows=cl, cl_cols=cl)
    counts = capi.dists_dense(gpu_ctx, db, out_mode=capi.OUT_COUNTS)
    np.testing.assert_array_equal(counts, oracle.dists(words, KMERS, S64, out_mode=2))
    jac = capi.dists_dense(gpu_ctx, db, random=rnd, out_mode=capi.OUT_JACCARD)
    np.testing.assert_array_equal(jac, oracle.dists(words, KMERS, S64, random=spec, out_mode=1))
    ca = capi.dists_dense(gpu_ctx, db, random=rnd)
    want = oracle.dists(words, KMERS, S64, random=spec)
    assert ca.shape == (2016, 2)
    np.testing.assert_allclose(ca, want, atol=1e-6, rtol=0)
    # the synthetic population spans the intended divergences
    assert 0.01 < np.median(ca[:, 0]) < 0.03 and ca[:, 0].max() < 0.05
    assert 0.05 < np.median(ca[:, 1]) < 0.3
