"""The floating-point error of every output, stated per output and per
workload (tests/fp_error.py holds the bars and the report): the genome case
sketched by the reference's own sketcher (64 x 2.5 Mb) under all three
random-match models, and the 4,096-sample bin-level all-vs-all."""
import json

import numpy as np
import pytest

import fp_error
import oracle
from sketchlib_b200 import capi

pytestmark = pytest.mark.gpu

KMERS = list(range(15, 31, 2))
S64 = 156


def _run(ctx, words, rnd=None, spec=None, kmers=KMERS):
    db = capi.Database(ctx, words, kmers, S64)
    if spec is not None and spec.mode == 1:
        db.set_sample_info(seq_len=spec.len_cols)
    if spec is not None and spec.mode == 2:
        db.set_sample_info(cluster=spec.cl_cols)
    jac = capi.dists_dense(ctx, db, random=rnd, out_mode=capi.OUT_JACCARD)
    ca = capi.dists_dense(ctx, db, random=rnd)
    db.close()
    want_j, f64, f32 = oracle.dists_multi(words, kmers, S64, random=spec)
    return jac, want_j, ca, f64, f32


@pytest.mark.skipif(not oracle.sketcher_available(), reason="reference sketcher not built")
@pytest.mark.parametrize("mode", ["none", "equal_base", "table"])
def test_fp_error_genomes(gpu_ctx, mode):
    rs = oracle.RefSketcher()
    words = rs.sketch(rs.genomes(64, 2_500_000, 0x5EED0001), KMERS, S64)
    rng = np.random.default_rng(1)
    rnd, spec = None, None
    if mode == "equal_base":
        lens = np.full(64, 2_500_000, np.uint64)
        rnd = capi.Random(gpu_ctx, capi.RANDOM_EQUAL_BASE, KMERS)
        spec = oracle.RandomSpec(1, True, len_rows=lens, len_cols=lens)
    elif mode == "table":
        cl = rng.integers(0, 3, 64).astype(np.uint16)
        table = rng.uniform(0, 0.003, (len(KMERS), 3, 3)).astype(np.float32)
        rnd = capi.Random(gpu_ctx, capi.RANDOM_TABLE, KMERS, table=table)
        spec = oracle.RandomSpec(2, True, table=table, cl_rows=cl, cl_cols=cl)
    rep = fp_error.check(*_run(gpu_ctx, words, rnd, spec))
    print("fp_error genomes", mode, json.dumps(rep))


def test_fp_error_4096_samples(gpu_ctx):
    """The whole 4,096-sample all-vs-all (8,386,560 pairs)."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))
    import bench
    words = bench.reference_inputs(threads=oracle.NTHREADS)
    rep = fp_error.check(*_run(gpu_ctx, words))
    assert rep["pairs"] == 4096 * 4095 // 2
    print("fp_error 4096", json.dumps(rep))
