"""The oracle's sketcher (sko_sketch, a restatement of the reference's
sketch(), src/sketch/sketch.cpp:120-168) pinned against golden vectors made by
the reference's own compiled sketcher (tests/golden/make_sketch_golden.py),
and against that sketcher directly where it was built."""
import numpy as np
import pytest

import oracle
from conftest import GOLDEN

G = np.load(GOLDEN / "sketch_golden.npz")


def reads_as_seqbuf(max_k):
    """The read set as the reference's SeqBuf holds it: upper case, reads
    shorter than the largest k dropped (src/sketch/seqio.cpp:67-87)."""
    b, off = G["reads_bases"], G["reads_seq_off"]
    seqs = [bytes(b[off[i]:off[i + 1]]).upper() for i in range(len(off) - 1)]
    return oracle.pack_samples([[q for q in seqs if len(q) >= max_k]])


@pytest.mark.parametrize("setting", [0, 1, 2, 3, 4])
def test_oracle_sketch_matches_reference_goldens(setting):
    kmers = G[f"seqs{setting}_kmers"]
    w, inv, dens = oracle.sketch(G["seqs_bases"], G["seqs_seq_off"], G["seqs_sample_seqs"], kmers,
                                 int(G[f"seqs{setting}_s64"]), bool(G[f"seqs{setting}_use_rc"]),
                                 codon_phased=bool(G[f"seqs{setting}_codon_phased"]))
    np.testing.assert_array_equal(w, G[f"seqs{setting}_words"])
    np.testing.assert_array_equal(inv, G[f"seqs{setting}_inv_minhash"])
    np.testing.assert_array_equal(dens, G[f"seqs{setting}_densified"])


@pytest.mark.parametrize("min_count", [2, 3])
def test_oracle_exact_count_matches_reference_goldens(min_count):
    kmers = G["reads_kmers"]
    bases, off, ss = reads_as_seqbuf(int(kmers.max()))
    w, inv, dens = oracle.sketch(bases, off, ss, kmers, int(G["reads_s64"]), True,
                                 min_count=min_count)
    np.testing.assert_array_equal(w[0], G[f"reads_mc{min_count}_words"])
    np.testing.assert_array_equal(inv[0], G[f"reads_mc{min_count}_inv_minhash"])
    assert bool(dens[0]) == bool(G[f"reads_mc{min_count}_densified"])
    # the filter is active: no filter (and the other threshold) give other sketches
    w0, _, _ = oracle.sketch(bases, off, ss, kmers, int(G["reads_s64"]), True)
    assert not np.array_equal(w0[0], w[0])


def test_golden_cases_cover_the_edges():
    dens = G["seqs0_densified"]
    assert dens.all()                      # 256 bins: every small sample has empty bins
    assert G["seqs2_densified"][3]         # all-N sample: densifybin returns -1, counted as densified
    ws = G["seqs1_words"]
    assert np.all(ws[3] == ~np.uint64(0))  # the all-N sample: every bin empty, all ones
    assert not np.array_equal(G["seqs0_words"][0], G["seqs0_words"][1])


@pytest.mark.skipif(not oracle.sketcher_available(), reason="oracle/_ref/libref_sketch.so not built")
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_sketch_matches_reference_random(seed):
    rng = np.random.default_rng(seed)
    alphabet = np.frombuffer(b"ACGTacgtNNRU", np.uint8)
    samples = []
    for _ in range(6):
        samples.append([alphabet[rng.integers(0, len(alphabet) if rng.random() < 0.3 else 4,
                                              int(rng.integers(1, 4000)))].tobytes()
                        for _ in range(int(rng.integers(1, 5)))])
    bases, off, ss = oracle.pack_samples(samples)
    kmers = sorted(rng.choice(np.arange(3, 80), 4, replace=False).tolist())
    s64 = int(rng.choice([1, 3, 16]))
    rc = bool(seed % 2)
    phased = seed == 3
    want = oracle.RefSketcher().sketch_seqs(bases, off, ss, kmers, s64, rc, codon_phased=phased)
    got = oracle.sketch(bases, off, ss, kmers, s64, rc, codon_phased=phased)
    for a, b in zip(got, want):
        np.testing.assert_array_equal(a, b)
