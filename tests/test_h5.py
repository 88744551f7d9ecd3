"""The built-in HDF5 reader (no libhdf5): sketch databases and random-match
tables written in the reference's on-disk layout read back exactly."""
from pathlib import Path

import os

import numpy as np
import pytest

import h5write
from conftest import GOLDEN

pp_sketchlib = pytest.importorskip("pp_sketchlib")

# the reference's own test databases, when its tree is named by PP_SKETCHLIB_REF
REF_TEST = Path(os.environ.get("PP_SKETCHLIB_REF", "/nonexistent")) / "test"


def _db(tmp_path, n=300, K=3, s64=16, random=None, seed=0):
    rng = np.random.default_rng(seed)
    names = [f"sample_{i:04d}" for i in range(n)]
    words = rng.integers(0, 2 ** 64, size=(n, K, s64 * 14), dtype=np.uint64)
    kmers = list(range(15, 15 + 2 * K, 2))
    lengths = rng.integers(1_000_000, 5_000_000, n)
    bases = rng.dirichlet(np.ones(4), n)
    path = tmp_path / "db"
    h5write.write_sketch_db(str(path) + ".h5", names, words, kmers, s64, lengths=lengths,
                            base_freq=bases, random=random)
    return str(path), names, words, kmers, lengths, bases


def test_sketches_roundtrip(tmp_path):
    path, names, words, kmers, lengths, bases = _db(tmp_path)
    got = pp_sketchlib._load_sketch_db(path, [], kmers)
    assert got["names"] == sorted(names)       # groups list in name order
    assert got["kmers"] == kmers and got["sketchsize64"] == 16 and got["bbits"] == 14
    order = [names.index(n) for n in got["names"]]
    np.testing.assert_array_equal(got["words"], words[order])
    np.testing.assert_array_equal(got["length"], lengths[order])
    np.testing.assert_allclose(got["base_freq"], bases[order], rtol=0, atol=0)
    # a subset of samples in the caller's order, k-mer lengths reordered
    pick = [names[7], names[3], names[250]]
    sub = pp_sketchlib._load_sketch_db(path, pick, [kmers[2], kmers[0]])
    assert sub["names"] == pick
    np.testing.assert_array_equal(sub["words"][:, 0], words[[7, 3, 250], 2])
    np.testing.assert_array_equal(sub["words"][:, 1], words[[7, 3, 250], 0])


def test_threaded_read_matches(tmp_path):
    """The multi-threaded read (what queryDatabase uses, straight from the
    mapped file into the caller's buffer) gives the single-threaded result,
    errors included."""
    path, names, words, kmers, lengths, bases = _db(tmp_path, n=257)
    one = pp_sketchlib._load_sketch_db(path, names, kmers, threads=1)
    many = pp_sketchlib._load_sketch_db(path, names, kmers, threads=8)
    np.testing.assert_array_equal(one["words"], words)
    np.testing.assert_array_equal(many["words"], words)
    assert many["length"] == one["length"] and many["base_freq"] == one["base_freq"]
    with pytest.raises(pp_sketchlib.HDF5Exception, match="Missing sketch"):
        pp_sketchlib._load_sketch_db(path, names[:100] + ["nope"] + names[100:], kmers, threads=8)


def test_missing_sample_and_kmer(tmp_path):
    path, names, *_ = _db(tmp_path, n=4)
    with pytest.raises(pp_sketchlib.HDF5Exception, match="Missing sketch"):
        pp_sketchlib._load_sketch_db(path, ["nope"], [15])
    with pytest.raises(RuntimeError, match="do not match those requested"):
        pp_sketchlib._load_sketch_db(path, names[:1], [15, 21])
    with pytest.raises(RuntimeError, match="Unable to open"):
        pp_sketchlib._load_sketch_db(str(tmp_path / "absent"), [], [15])


def test_random_table_roundtrip(tmp_path):
    C = 3
    rng = np.random.default_rng(2)
    table_names = [f"sample_{i:04d}" for i in range(0, 20, 2)]
    rand = dict(k_min=6, k_max=30, use_rc=1,
                table={n: i % C for i, n in enumerate(table_names)},
                matches={k: rng.uniform(0, 1 if k > 6 else 2, (C, C)).astype(np.float32)
                         for k in range(6, 31)},
                centroids=rng.dirichlet(np.ones(4), C).astype(np.float32))
    path, *_ = _db(tmp_path, n=20, random=rand)
    r = pp_sketchlib._load_random(path)
    assert r["mode"] == 2 and r["k_min"] == 6 and r["k_max"] == 30 and r["n_clusters"] == C
    assert r["cluster_table"] == rand["table"]
    for k, m in rand["matches"].items():
        np.testing.assert_array_equal(np.asarray(r["matches"][k], np.float32), m.ravel())
    np.testing.assert_array_equal(np.asarray(r["centroids"], np.float32), rand["centroids"].ravel())
    # min_supported_k: first k from k_min whose mean random match is below 1
    means = {k: float(np.mean(m.astype(np.float64))) for k, m in rand["matches"].items()}
    assert r["min_supported_k"] == next(k for k in range(6, 30) if means[k] < 1)


def test_no_random_group_means_equal_base(tmp_path):
    path, *_ = _db(tmp_path, n=3)
    assert pp_sketchlib._load_random(path)["mode"] == 1


@pytest.mark.skipif(not (REF_TEST / "small_mass_plus1.h5").exists(),
                    reason="reference test databases not present")
def test_reads_reference_databases():
    fx = np.load(GOLDEN / "small_mass_sketches.npz")
    kmers = [int(k) for k in fx["kmers"]]
    got = pp_sketchlib._load_sketch_db(str(REF_TEST / "small_mass_plus1"), [], kmers)
    assert got["names"] == list(fx["names"])
    np.testing.assert_array_equal(got["words"], fx["words"])
    small = pp_sketchlib._load_sketch_db(str(REF_TEST / "small_mass"), [], kmers)
    assert len(small["names"]) == int(fx["n_small"])


def test_reference_fixture_is_sane():
    """The extracted real sketches behave like sketches: a sample matches itself
    in every bin and related samples share far more bins than chance."""
    import oracle
    fx = np.load(GOLDEN / "small_mass_sketches.npz")
    w = fx["words"]
    assert w.shape == (7, 6, 156 * 14)
    assert oracle.intersize(w[0, 0], w[0, 0], 156) == 64 * 156
    c = oracle.intersize(w[0, 0], w[1, 0], 156)
    assert c > 64 * 156 * 0.05
