"""Outputs larger than the device memory allowed for them are computed in
blocks of row tiles and copied back while the next block computes (the
reference chunks an all-vs-all that exceeds device memory,
src/gpu/gpu_api.cpp:357-389).  Blocked results must be bit-identical to the
one-shot results, whatever the block size."""
import numpy as np
import pytest

from conftest import random_sketches
from sketchlib_b200 import capi

pytestmark = pytest.mark.gpu


@pytest.fixture
def limited(gpu_ctx):
    yield gpu_ctx
    gpu_ctx.set_memory_limit(0)
    gpu_ctx.set_semantics(capi.SEMANTICS_REFERENCE_CPU)


@pytest.mark.parametrize("limit", [1, 40_000, 700_000])     # one row tile per block .. a few blocks
@pytest.mark.parametrize("mode", [capi.OUT_CORE_ACC, capi.OUT_JACCARD, capi.OUT_COUNTS])
def test_self_blocked_equals_one_shot(limited, limit, mode):
    words, kmers = random_sketches(1000, 4, 32, seed=1201)
    rng = np.random.default_rng(3)
    cl = rng.integers(0, 2, 1000).astype(np.uint16)
    table = rng.uniform(0, 0.01, (4, 2, 2)).astype(np.float32)
    rnd = capi.Random(limited, capi.RANDOM_TABLE, kmers, table=table)
    db = capi.Database(limited, words, kmers, 32, cluster=cl)
    want = capi.dists_dense(limited, db, random=rnd, out_mode=mode)
    limited.set_memory_limit(limit)
    got = capi.dists_dense(limited, db, random=rnd, out_mode=mode)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("semantics", [capi.SEMANTICS_REFERENCE_CPU, capi.SEMANTICS_REFERENCE_GPU])
def test_query_blocked_equals_one_shot(limited, semantics):
    words, kmers = random_sketches(1033, 5, 16, seed=1202)
    rw, qw = words[333:], words[:333]
    limited.set_semantics(semantics)
    ref = capi.Database(limited, rw, kmers, 16)
    qry = capi.Database(limited, qw, kmers, 16)
    want = capi.dists_dense(limited, ref, qry)
    limited.set_memory_limit(100_000)
    np.testing.assert_array_equal(capi.dists_dense(limited, ref, qry), want)
    # the pipelined host call falls back to the blocked computation too
    np.testing.assert_array_equal(capi.query_db(limited, rw, kmers, 16, query_words=qw), want)


def test_query_db_blocked_self_and_pinned(limited):
    import torch
    words, kmers = random_sketches(1500, 3, 16, seed=1203)
    want = capi.query_db(limited, words, kmers, 16)
    limited.set_memory_limit(250_000)
    out = torch.empty(want.shape, dtype=torch.float32).pin_memory().numpy()
    got = capi.query_db(limited, words, kmers, 16, out=out)
    np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(capi.query_db(limited, words, kmers, 16), want)   # pageable


def test_negative_limit_refused(gpu_ctx):
    with pytest.raises(capi.SketchlibError):
        gpu_ctx.set_memory_limit(-1)
