"""Batched persistent launch (one graph-captured launch over many uneven jobs)
against the plain single-job path, pair for pair, and against the oracle;
tail splitting along k against unsplit tiles; the autotuner."""
import numpy as np
import pytest

import oracle
from conftest import random_sketches
from sketchlib_b200 import capi

pytestmark = pytest.mark.gpu


def _width(mode, K):
    return 2 if mode == capi.OUT_CORE_ACC else K


def _dtype(mode):
    return np.uint32 if mode == capi.OUT_COUNTS else np.float32


def _job_specs():
    # (n_ref, n_query or None, K, s64, out_mode, random)
    return [
        (700, None, 8, 156, capi.OUT_CORE_ACC, "none"),
        (50, None, 4, 16, capi.OUT_JACCARD, "equal_base"),
        (300, 40, 14, 64, capi.OUT_CORE_ACC, "table"),
        (129, None, 5, 312, capi.OUT_COUNTS, "none"),
        (1000, 3, 8, 156, capi.OUT_CORE_ACC, "equal_base"),
        (64, 64, 11, 16, capi.OUT_JACCARD, "none"),
        (257, None, 6, 64, capi.OUT_CORE_ACC, "table"),
        # the batched workload's widest shape: K = 14 over k = 13..39 at
        # sketch_size 20,000 (sketchsize64 312), self and query
        (400, None, 14, 312, capi.OUT_CORE_ACC, "equal_base"),
        (350, 60, 14, 312, capi.OUT_CORE_ACC, "table"),
        (200, 30, 14, 312, capi.OUT_JACCARD, "none"),
        (330, None, 14, 312, capi.OUT_COUNTS, "table"),
    ]


def _make(ctx, spec, seed):
    import torch
    n, nq, K, s64, mode, rmode = spec
    w, _ = random_sketches(n + (nq or 0), K, s64, seed=seed)
    kmers = np.arange(13, 13 + 2 * K, 2, dtype=np.int32)
    rng = np.random.default_rng(seed)
    lens = rng.integers(1_000_000, 6_000_000, n + (nq or 0)).astype(np.uint64)
    cl = rng.integers(0, 3, n + (nq or 0)).astype(np.uint16)
    ref = capi.Database(ctx, w[:n], kmers, s64, cluster=cl[:n], seq_len=lens[:n])
    qry = None if nq is None else capi.Database(ctx, w[n:], kmers, s64, cluster=cl[n:],
                                                 seq_len=lens[n:])
    rnd, spec_o = None, None
    rows_sl = slice(0, n) if nq is None else slice(n, n + nq)
    if rmode == "equal_base":
        rnd = capi.Random(ctx, capi.RANDOM_EQUAL_BASE, kmers)
        spec_o = oracle.RandomSpec(mode=1, len_rows=lens[rows_sl], len_cols=lens[:n])
    elif rmode == "table":
        table = rng.uniform(0, 0.01, (K, 3, 3)).astype(np.float32)
        rnd = capi.Random(ctx, capi.RANDOM_TABLE, kmers, table=table)
        spec_o = oracle.RandomSpec(mode=2, table=table, cl_rows=cl[rows_sl], cl_cols=cl[:n])
    rows = capi.dists_rows(ref, qry)
    tdt = torch.int32 if mode == capi.OUT_COUNTS else torch.float32
    out = torch.full((max(rows, 1), _width(mode, K)), -7, dtype=tdt, device="cuda")
    want = oracle.dists(w[:n], kmers, s64, query_words=None if nq is None else w[n:],
                        random=spec_o, out_mode=mode)
    return (ref, qry, rnd, mode, out), want


def test_batch_equals_plain_and_oracle(gpu_ctx):
    """Every job of one batched launch equals the plain single-job path pair
    for pair and the oracle: counts and Jaccards exactly, core/accessory
    within 1e-6 of its double fit (tolerance per database: 5 / (64 s64))."""
    specs = _job_specs()
    made, wants = zip(*[_make(gpu_ctx, sp, 100 + i) for i, sp in enumerate(specs)])
    batch = capi.Batch(gpu_ctx, [(r, q, rnd, m, o.data_ptr()) for r, q, rnd, m, o in made])
    info = batch.info()
    assert info["n_pairs"] == sum(capi.dists_rows(r, q) for r, q, *_ in made)
    for rep in range(2):            # graph replay gives the same results
        for *_, o in made:
            o.fill_(-7)
        batch.run()
        for (ref, qry, rnd, mode, out), want, sp in zip(made, wants, specs):
            plain = capi.dists_dense(gpu_ctx, ref, qry, rnd, out_mode=mode)
            got = out.cpu().numpy()[: plain.shape[0]]
            if mode == capi.OUT_COUNTS:
                got = got.view(np.uint32)
            np.testing.assert_array_equal(got, plain, err_msg=f"job {sp} replay {rep}")
            if mode == capi.OUT_CORE_ACC:
                np.testing.assert_allclose(got, want, rtol=0, atol=1e-6, err_msg=f"job {sp}")
            else:
                np.testing.assert_array_equal(got, want, err_msg=f"job {sp}")
    batch.close()


@pytest.mark.parametrize("n", [300, 1100, 2300])
def test_tail_split_matches_oracle(gpu_ctx, n):
    """Sizes whose last wave is split along k (tiles not a multiple of the
    resident CTAs) give the oracle's counts exactly."""
    w, kmers = random_sketches(n, 8, 16, seed=n)
    db = capi.Database(gpu_ctx, w, kmers, 16)
    got = capi.dists_dense(gpu_ctx, db, out_mode=capi.OUT_COUNTS)
    np.testing.assert_array_equal(got, oracle.dists(w, kmers, 16, out_mode=2))
    ca = capi.dists_dense(gpu_ctx, db)
    np.testing.assert_allclose(ca, oracle.dists(w, kmers, 16), atol=1e-6, rtol=0)


def test_autotune_and_tuning_table(gpu_ctx, tmp_path):
    w, kmers = random_sketches(600, 8, 156, seed=4)
    db = capi.Database(gpu_ctx, w, kmers, 156)
    best = capi.autotune(gpu_ctx, db, repeats=1)
    assert 1 <= best <= len(capi.tile_configs())
    path = tmp_path / "tuning.txt"
    capi.save_tuning(gpu_ctx, path)
    assert f"8 156 {best}" in path.read_text()
    gpu_ctx.load_tuning(path)
    np.testing.assert_array_equal(capi.dists_dense(gpu_ctx, db, out_mode=capi.OUT_COUNTS),
                                  oracle.dists(w, kmers, 156, out_mode=2))
    # a batch with the autotune flag picks a shape by timing the batch itself
    import torch
    out = torch.empty((600 * 599 // 2, 2), dtype=torch.float32, device="cuda")
    b = capi.Batch(gpu_ctx, [(db, None, None, capi.OUT_CORE_ACC, out.data_ptr())], autotune=True)
    b.run()
    np.testing.assert_array_equal(out.cpu().numpy(), capi.dists_dense(gpu_ctx, db))
    b.close()
