"""The CUDA path against the reference's own GPU kernel.

`calculate_dists` (src/gpu/dist.cu:164-317) is compiled for sm_100a from the
reference sources into oracle/_ref/libref_gpu.so and launched the way the
reference's dispatchDists does.  It is a second witness, not the oracle: it
regresses in float with round-up intrinsics and stops at the first k whose
Jaccard falls below the tolerance, where the reference's CPU path (which this
library follows) fits the range between the first and last k above it.  So
the bar is the reference's own GPU-vs-CPU rule (test/gpu_test.py:14-30: a
value fails when it differs by more than 1e-3 absolute AND 5% relative, or
when exactly one side is zero), applied to the pairs for which both
truncation rules select the same k points.  Pairs whose selected Jaccards
are all equal are left out too: there the reference kernel's correlation form
(src/gpu/dist.cu:105-110) divides 0 by 0 and writes (0, 0), where the CPU fit
gives slope 0 and accessory 1 - J.
"""
import numpy as np
import pytest

import oracle

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.ref_gpu_available(),
                                 reason="oracle/_ref/libref_gpu.so not built")]

MAX_DIFF, MAX_FRAC = 1e-3, 0.05          # test/gpu_test.py:16-17


def same_points(jac, s64, margin=1e-6):
    """Pairs whose CPU range rule and GPU prefix rule pick the same k, with
    every Jaccard at least `margin` away from the tolerance."""
    tol = 5.0 / (64 * s64)
    above = jac > tol
    near = np.abs(jac - tol) <= margin * max(tol, 1.0)
    K = jac.shape[1]
    idx = np.arange(K)
    first_low = np.where(~above, idx, K).min(axis=1)           # GPU: prefix before the first low k
    gpu_set = idx[None, :] < first_low[:, None]
    any_above = above.any(axis=1)
    first = np.where(above, idx, K).min(axis=1)
    last = np.where(above, idx, -1).max(axis=1)
    cpu_set = (idx[None, :] >= first[:, None]) & (idx[None, :] <= last[:, None]) & any_above[:, None]
    zero_inside = (cpu_set & (jac <= 0)).any(axis=1)
    sel_max = np.where(cpu_set, jac, -np.inf).max(axis=1)
    sel_min = np.where(cpu_set, jac, np.inf).min(axis=1)
    flat = (cpu_set.sum(axis=1) >= 2) & (sel_max == sel_min)
    return (gpu_set == cpu_set).all(axis=1) & ~near.any(axis=1) & ~zero_inside & ~flat


def failures(ours, ref):
    d = ours.astype(np.float64) - ref.astype(np.float64)
    s = ours.astype(np.float64) + ref.astype(np.float64)
    frac = np.divide(2 * d, s, out=np.zeros_like(d), where=s != 0)
    both = (ours != 0) & (ref != 0)
    bad = both & (np.abs(d) > MAX_DIFF) & (np.abs(frac) > MAX_FRAC)
    bad |= (ours == 0) != (ref == 0)
    return bad


def compare(gpu_ctx, words, kmers, s64, random_k=None):
    from sketchlib_b200 import capi
    K = len(kmers)
    n = words.shape[0]
    db = capi.Database(gpu_ctx, words, kmers, s64)
    if random_k is None:
        rnd, spec = None, oracle.RandomSpec()
    else:
        table = np.asarray(random_k, np.float32).reshape(K, 1, 1)
        rnd = capi.Random(gpu_ctx, capi.RANDOM_TABLE, kmers, table=table)
        zeros = np.zeros(n, np.uint16)
        spec = oracle.RandomSpec(2, True, table=table, cl_rows=zeros, cl_cols=zeros)
    ours = capi.dists_dense(gpu_ctx, db, random=rnd)
    ref, _ = oracle.RefGpuKernel().self_dists(words, kmers, s64, random_k=random_k)
    jac = oracle.dists(words, kmers, s64, random=spec, out_mode=1).astype(np.float64)
    keep = same_points(jac, s64)
    bad = failures(ours, ref) & keep[:, None]
    return ours, ref, keep, bad


def test_reference_gpu_kernel_on_reference_sketches(gpu_ctx):
    """64 genomes sketched by the reference's own sketcher."""
    if not oracle.sketcher_available():
        pytest.skip("oracle/_ref/libref_sketch.so not built")
    kmers = list(range(15, 31, 2))
    rs = oracle.RefSketcher()
    words = rs.sketch(rs.genomes(64, 2_500_000, 0x5EED0001), kmers, 156)
    ours, ref, keep, bad = compare(gpu_ctx, words, kmers, 156)
    assert keep.mean() > 0.99
    assert not bad.any(), np.argwhere(bad)[:10]
    # both are float fits of the same points: close well inside the bar
    assert np.quantile(np.abs(ours[keep] - ref[keep]), 0.99) < 1e-4


@pytest.mark.parametrize("random_k,c_max,min_keep", [(None, 0.03, 0.85), ("table", 0.01, 0.99)])
def test_reference_gpu_kernel_on_synthetic_tree(gpu_ctx, random_k, c_max, min_keep):
    from sketchlib_b200 import capi, synth
    kmers = [13, 17, 21, 25, 29, 33]
    s64 = 64
    parent, thresh = synth.random_tree(300, kmers=kmers, seed=0x5EED00A1, c_max=c_max)
    words = capi.synth_host(parent, thresh, s64, seed=0x5EED00A1)
    rk = None if random_k is None else np.linspace(0.004, 0.0005, len(kmers)).astype(np.float32)
    ours, ref, keep, bad = compare(gpu_ctx, words, kmers, s64, random_k=rk)
    assert keep.mean() > min_keep
    assert not bad.any(), np.argwhere(bad)[:10]


# ---------------------------------------------------------------------------
# SK_SEMANTICS_REFERENCE_GPU: the same kernel with the reference GPU path's
# arithmetic must give the reference kernel's output bit for bit, including
# the pairs the CPU semantics treat differently (first-low-k truncation,
# equal Jaccards, float rounding).

@pytest.fixture
def gpu_semantics(gpu_ctx):
    from sketchlib_b200 import capi
    gpu_ctx.set_semantics(capi.SEMANTICS_REFERENCE_GPU)
    yield gpu_ctx
    gpu_ctx.set_semantics(capi.SEMANTICS_REFERENCE_CPU)


def _synthetic(n, kmers, s64, seed, c_max=0.03):
    from sketchlib_b200 import capi, synth
    parent, thresh = synth.random_tree(n, kmers=kmers, seed=seed, c_max=c_max)
    return capi.synth_host(parent, thresh, s64, seed=seed)


def test_gpu_semantics_bit_identical_on_reference_sketches(gpu_semantics):
    from sketchlib_b200 import capi
    if not oracle.sketcher_available():
        pytest.skip("oracle/_ref/libref_sketch.so not built")
    kmers = list(range(15, 31, 2))
    rs = oracle.RefSketcher()
    words = rs.sketch(rs.genomes(64, 2_500_000, 0x5EED0001), kmers, 156)
    db = capi.Database(gpu_semantics, words, kmers, 156)
    np.testing.assert_array_equal(capi.dists_dense(gpu_semantics, db),
                                  oracle.RefGpuKernel().dists(words, kmers, 156))


@pytest.mark.parametrize("kind", ["none", "equal_base", "table"])
def test_gpu_semantics_bit_identical_self(gpu_semantics, kind):
    from sketchlib_b200 import capi
    kmers = [13, 17, 21, 25, 29, 33]
    words = _synthetic(300, kmers, 64, 0x5EED00A1)     # includes truncated and flat pairs
    n = words.shape[0]
    rng = np.random.default_rng(5)
    lens = rng.integers(1_000_000, 6_000_000, n).astype(np.uint64)
    cl = rng.integers(0, 3, n).astype(np.uint16)
    table = rng.uniform(0, 0.02, (len(kmers), 3, 3)).astype(np.float32)
    if kind == "none":
        rnd, witness = None, {}
    elif kind == "equal_base":
        rnd = capi.Random(gpu_semantics, capi.RANDOM_EQUAL_BASE, kmers)
        per_k = np.array([oracle.csrs(k, True, int(lens[0]), int(lens[0])) for k in kmers], np.float32)
        witness = dict(table=per_k)
    else:
        rnd = capi.Random(gpu_semantics, capi.RANDOM_TABLE, kmers, table=table)
        witness = dict(table=table, ref_lookup=cl)
    db = capi.Database(gpu_semantics, words, kmers, 64, cluster=cl, seq_len=lens)
    got = capi.dists_dense(gpu_semantics, db, random=rnd)
    want = oracle.RefGpuKernel().dists(words, kmers, 64, **witness)
    np.testing.assert_array_equal(got, want)
    # the CPU semantics differ on some of these pairs: the comparison has teeth
    gpu_semantics.set_semantics(capi.SEMANTICS_REFERENCE_CPU)
    assert np.any(capi.dists_dense(gpu_semantics, db, random=rnd) != want)


@pytest.mark.parametrize("kind", ["none", "table"])
def test_gpu_semantics_bit_identical_query(gpu_semantics, kind):
    from sketchlib_b200 import capi
    kmers = [15, 19, 23, 27, 31]
    words = _synthetic(900, kmers, 32, 0x5EED00A2)
    qw, rw = words[:150], words[150:]
    rng = np.random.default_rng(6)
    rcl = rng.integers(0, 4, rw.shape[0]).astype(np.uint16)
    qcl = rng.integers(0, 4, qw.shape[0]).astype(np.uint16)
    table = rng.uniform(0, 0.02, (len(kmers), 4, 4)).astype(np.float32)
    rnd = None if kind == "none" else capi.Random(gpu_semantics, capi.RANDOM_TABLE, kmers, table=table)
    witness = {} if kind == "none" else dict(table=table, ref_lookup=rcl, query_lookup=qcl)
    ref = capi.Database(gpu_semantics, rw, kmers, 32, cluster=rcl)
    qry = capi.Database(gpu_semantics, qw, kmers, 32, cluster=qcl)
    got = capi.dists_dense(gpu_semantics, ref, qry, random=rnd)
    want = oracle.RefGpuKernel().dists(rw, kmers, 32, query_words=qw, **witness)
    np.testing.assert_array_equal(got, want)
    # the pipelined host-to-host call follows the same semantics
    got2 = capi.query_db(gpu_semantics, rw, kmers, 32, query_words=qw, ref_cluster=rcl,
                         query_cluster=qcl, random=rnd)
    np.testing.assert_array_equal(got2, want)


def test_gpu_semantics_knn(gpu_semantics):
    """kNN under GPU semantics ranks the reference kernel's distances."""
    from sketchlib_b200 import capi
    kmers = [13, 17, 21, 25, 29, 33]
    words = _synthetic(300, kmers, 64, 0x5EED00A3)
    n = words.shape[0]
    db = capi.Database(gpu_semantics, words, kmers, 64)
    want = oracle.RefGpuKernel().dists(words, kmers, 64)
    i, j, d = capi.dists_knn(gpu_semantics, db, 5, dist_col=1)
    sq = np.full((n, n), np.inf)
    iu = np.triu_indices(n, 1)
    sq[iu] = want[:, 1]
    sq[(iu[1], iu[0])] = want[:, 1]
    order = np.lexsort((np.tile(np.arange(n), (n, 1)), sq), axis=1)[:, :5]
    np.testing.assert_array_equal(j.reshape(n, 5), order)
    np.testing.assert_array_equal(d.reshape(n, 5), np.take_along_axis(sq, order, 1).astype(np.float32))
