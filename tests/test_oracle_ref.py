"""Checks the oracle's restatement against the reference's own compiled code
(oracle/_ref: src/dist/dist.cpp built from the reference sources).  Skipped
where that build is absent."""
import numpy as np
import pytest

import oracle
from conftest import random_sketches

pytestmark = pytest.mark.skipif(not oracle.ref_available(),
                                reason="oracle/_ref not built (needs the reference sources)")


@pytest.mark.parametrize("s64", [1, 2, 16, 156, 312])
def test_intersize_matches_reference(s64):
    ref = oracle.RefQueryDb()
    rng = np.random.default_rng(s64)
    for trial in range(20):
        a = rng.integers(0, 2 ** 64, size=s64 * 14, dtype=np.uint64)
        b = a.copy()
        # flip a random subset of planes so some bins match and some do not
        flips = rng.integers(0, 2 ** 64, size=s64 * 14, dtype=np.uint64)
        mask = rng.random(s64 * 14) < rng.random()
        b[mask] ^= flips[mask]
        assert oracle.intersize(a, b, s64) == ref.intersize(a, b, s64)
        assert oracle.intersize(a, a, s64) == 64 * s64


def test_query_db_loop_matches_reference():
    words, kmers = random_sketches(40, 8, 156, seed=11)
    ref = oracle.RefQueryDb()
    ref_out, done = ref.self_dists(words, kmers, 156, threads=4)
    assert done == 40 * 39 // 2
    f32 = oracle.dists(words, kmers, 156, regress=1, threads=4)
    np.testing.assert_array_equal(oracle.dists(words, kmers, 156, out_mode=2)[:, 0],
                                  oracle.dists(words, kmers, 156, out_mode=2)[:, 0])
    # same counts, same float arithmetic apart from the reference's -ffast-math
    assert np.abs(ref_out - f32).max() < 1e-5
    f64 = oracle.dists(words, kmers, 156, regress=0, threads=4)
    assert np.abs(ref_out - f64).max() < 1e-5


@pytest.mark.skipif(not oracle.ref_gpu_available(), reason="oracle/_ref/libref_gpu.so not built")
def test_reference_gpu_harness_loads():
    """The reference GPU kernel harness loads on a host without a GPU (its
    launches run only in the GPU tests and the reference arm of the bench)."""
    k = oracle.RefGpuKernel()
    assert hasattr(k.lib, "refgpu_self_dists")

