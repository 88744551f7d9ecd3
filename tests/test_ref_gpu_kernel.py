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
