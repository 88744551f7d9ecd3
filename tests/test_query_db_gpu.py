"""sk_query_db: host sketches in, host distances out, with the upload chunked
and overlapped with the distance kernel.  Its results must be bit-identical to
sk_db_create + sk_dists_dense (the same kernel on the same tiles, only
scheduled per chunk) for every output mode, random model and chunk layout,
and equal to the oracle."""
import numpy as np
import pytest

import oracle
from conftest import random_sketches
from sketchlib_b200 import capi

pytestmark = pytest.mark.gpu

MODES = [capi.OUT_CORE_ACC, capi.OUT_JACCARD, capi.OUT_COUNTS]


def _random(ctx, kind, kmers, n_ref, n_q, seed):
    rng = np.random.default_rng(seed)
    info = dict(ref_cluster=None, ref_seq_len=None, query_cluster=None, query_seq_len=None)
    if kind == "none":
        return None, info
    if kind == "equal_base":
        info["ref_seq_len"] = rng.integers(1_000_000, 6_000_000, n_ref).astype(np.uint64)
        info["query_seq_len"] = rng.integers(1_000_000, 6_000_000, n_q).astype(np.uint64)
        return capi.Random(ctx, capi.RANDOM_EQUAL_BASE, kmers), info
    C = 3
    table = rng.uniform(0, 0.01, (len(kmers), C, C)).astype(np.float32)
    info["ref_cluster"] = rng.integers(0, C, n_ref).astype(np.uint16)
    info["query_cluster"] = rng.integers(0, C, n_q).astype(np.uint16)
    return capi.Random(ctx, capi.RANDOM_TABLE, kmers, table=table), info


def _plain(ctx, words, kmers, s64, qwords, rnd, info, mode):
    ref = capi.Database(ctx, words, kmers, s64, cluster=info["ref_cluster"],
                        seq_len=info["ref_seq_len"])
    qry = None
    if qwords is not None:
        qry = capi.Database(ctx, qwords, kmers, s64, cluster=info["query_cluster"],
                            seq_len=info["query_seq_len"])
    return capi.dists_dense(ctx, ref, qry, rnd, out_mode=mode)


@pytest.mark.parametrize("n", [70, 1300, 2600])          # 1, 3 and 6 upload chunks
@pytest.mark.parametrize("kind", ["none", "equal_base", "table"])
def test_self_matches_plain_path(gpu_ctx, n, kind):
    words, kmers = random_sketches(n, 3, 16, seed=900 + n)
    rnd, info = _random(gpu_ctx, kind, kmers, n, 0, seed=n)
    import torch
    for mode in MODES:
        got = capi.query_db(gpu_ctx, words, kmers, 16, ref_cluster=info["ref_cluster"],
                            ref_seq_len=info["ref_seq_len"], random=rnd, out_mode=mode)
        want = _plain(gpu_ctx, words, kmers, 16, None, rnd, info, mode)
        np.testing.assert_array_equal(got, want)
        # a pinned destination takes each chunk's rows back as soon as they are final
        pinned = torch.zeros(want.shape, dtype=torch.float32 if want.dtype == np.float32
                             else torch.int32).pin_memory().numpy().view(want.dtype)
        got2 = capi.query_db(gpu_ctx, words, kmers, 16, ref_cluster=info["ref_cluster"],
                             ref_seq_len=info["ref_seq_len"], random=rnd, out_mode=mode, out=pinned)
        np.testing.assert_array_equal(got2, want)


@pytest.mark.parametrize("n_ref,n_q", [(1100, 300), (600, 1), (70, 700)])
@pytest.mark.parametrize("kind", ["none", "table"])
def test_query_matches_plain_path(gpu_ctx, n_ref, n_q, kind):
    words, kmers = random_sketches(n_ref + n_q, 4, 8, seed=n_ref * 3 + n_q)
    rw, qw = words[n_q:], words[:n_q]
    rnd, info = _random(gpu_ctx, kind, kmers, n_ref, n_q, seed=n_q)
    for mode in (capi.OUT_CORE_ACC, capi.OUT_COUNTS):
        got = capi.query_db(gpu_ctx, rw, kmers, 8, query_words=qw, random=rnd, out_mode=mode, **info)
        want = _plain(gpu_ctx, rw, kmers, 8, qw, rnd, info, mode)
        np.testing.assert_array_equal(got, want)


def test_against_oracle_and_pinned_buffers(gpu_ctx):
    import torch
    words, kmers = random_sketches(1400, 8, 156, seed=4242)
    pinned = torch.from_numpy(words.view(np.int64)).pin_memory().numpy().view(np.uint64)
    out = torch.empty((1400 * 1399 // 2, 2), dtype=torch.float32).pin_memory().numpy()
    got = capi.query_db(gpu_ctx, pinned, kmers, 156, out=out)
    assert got is out
    np.testing.assert_array_equal(capi.query_db(gpu_ctx, words, kmers, 156), got)
    counts = capi.query_db(gpu_ctx, pinned, kmers, 156, out_mode=capi.OUT_COUNTS)
    np.testing.assert_array_equal(counts, oracle.dists(words, kmers, 156, out_mode=2))
    np.testing.assert_allclose(got, oracle.dists(words, kmers, 156), atol=1e-6, rtol=0)


def test_empty_and_single_sample(gpu_ctx):
    """The reference refuses empty lists ("Query with empty ref or query
    list!", src/api.cpp:146); one sample all-vs-all has no pairs."""
    words, kmers = random_sketches(5, 2, 4, seed=3)
    assert capi.query_db(gpu_ctx, words[:1], kmers, 4).shape == (0, 2)
    for bad in (dict(ref_words=words[:0]), dict(ref_words=words, query_words=words[:0])):
        with pytest.raises(capi.SketchlibError, match="empty ref or query"):
            capi.query_db(gpu_ctx, kmers=kmers, sketchsize64=4, **bad)
    with pytest.raises(capi.SketchlibError):
        capi.query_db(gpu_ctx, words, kmers, 4, bbits=13)


@pytest.mark.parametrize("self_", [True, False])
def test_words_filled_while_the_call_runs(gpu_ctx, self_):
    """sk_query_db_ready: the words start as zeros and a thread copies them in,
    chunk by chunk in the order the call asks for them, only when asked; the
    result equals the call on complete words, and every sample was asked for
    exactly once before its words were read."""
    import threading
    words, kmers = random_sketches(2600, 4, 16, seed=77)
    qwords = None if self_ else words[:300].copy()
    rwords = words if self_ else words[300:].copy()
    want = capi.query_db(gpu_ctx, rwords, kmers, 16, query_words=qwords)
    sides = [np.zeros_like(rwords), None if self_ else np.zeros_like(qwords)]
    srcs = [rwords, qwords]
    asked = [np.zeros(len(rwords), np.int32), None if self_ else np.zeros(len(qwords), np.int32)]
    order = []

    def ready(side, s0, n):
        order.append((side, s0, n))
        asked[side][s0:s0 + n] += 1
        done = threading.Event()

        def fill():
            sides[side][s0:s0 + n] = srcs[side][s0:s0 + n]
            done.set()
        threading.Thread(target=fill).start()
        return done.wait(30)

    got = capi.query_db(gpu_ctx, sides[0], kmers, 16, query_words=sides[1], ready=ready)
    np.testing.assert_array_equal(got, want)
    assert all((a == 1).all() for a in asked if a is not None)
    if self_:      # all-vs-all: from the last samples down
        assert [s0 for _, s0, _ in order] == sorted((s0 for _, s0, _ in order), reverse=True)
    else:          # the queries first, then the references from the first up
        assert [side for side, _, _ in order][:1] == [1] and order[-1][0] == 0


def test_words_never_ready_abandons_the_call(gpu_ctx):
    words, kmers = random_sketches(1300, 4, 16, seed=78)
    with pytest.raises(capi.SketchlibError, match="never became ready"):
        capi.query_db(gpu_ctx, words, kmers, 16, ready=lambda side, s0, n: s0 > 600)
    # the context still serves calls
    np.testing.assert_array_equal(capi.query_db(gpu_ctx, words, kmers, 16),
                                  capi.query_db(gpu_ctx, words, kmers, 16))
