"""Sketching on the device (sk_sketch) against the reference's sketcher: the
golden vectors of tests/golden/sketch_golden.npz (made by the reference's own
sketch()), the oracle's restatement on seeded random inputs, and the
reference's compiled sketcher at the 64-genome size where it was built."""
import numpy as np
import pytest

import oracle
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

G = np.load(GOLDEN / "sketch_golden.npz")


def check(got, want):
    for a, b in zip(got, want):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("setting", [0, 1, 2, 3, 4])
def test_sketch_matches_reference_goldens(gpu_ctx, setting):
    from sketchlib_b200 import capi
    got = capi.sketch(gpu_ctx, G["seqs_bases"], G["seqs_seq_off"], G["seqs_sample_seqs"],
                      G[f"seqs{setting}_kmers"], int(G[f"seqs{setting}_s64"]),
                      use_rc=bool(G[f"seqs{setting}_use_rc"]),
                      codon_phased=bool(G[f"seqs{setting}_codon_phased"]))
    check(got, (G[f"seqs{setting}_words"], G[f"seqs{setting}_inv_minhash"],
                G[f"seqs{setting}_densified"]))


@pytest.mark.parametrize("min_count", [2, 3])
def test_read_filter_matches_reference_goldens(gpu_ctx, min_count):
    from sketchlib_b200 import capi
    kmers = G["reads_kmers"]
    b, off = G["reads_bases"], G["reads_seq_off"]
    seqs = [bytes(b[off[i]:off[i + 1]]).upper() for i in range(len(off) - 1)]
    bases, so, ss = capi.pack_sequences([[q for q in seqs if len(q) >= kmers.max()]])
    w, inv, dens = capi.sketch(gpu_ctx, bases, so, ss, kmers, int(G["reads_s64"]),
                               min_count=min_count)
    np.testing.assert_array_equal(w[0], G[f"reads_mc{min_count}_words"])
    np.testing.assert_array_equal(inv[0], G[f"reads_mc{min_count}_inv_minhash"])
    assert bool(dens[0]) == bool(G[f"reads_mc{min_count}_densified"])


def random_samples(rng, n, max_len, n_frac=0.3, max_seqs=4):
    alphabet = np.frombuffer(b"ACGTacgtNNRUu", np.uint8)
    out = []
    for _ in range(n):
        smp = []
        for _ in range(int(rng.integers(1, max_seqs + 1))):
            L = int(rng.integers(0, max_len))
            a = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, L)].copy()
            if rng.random() < n_frac:
                m = rng.random(L) < 0.002
                a[m] = alphabet[rng.integers(0, len(alphabet), int(m.sum()))]
            smp.append(a.tobytes())
        out.append(smp)
    return out


@pytest.mark.parametrize("seed,kmers,s64,rc", [
    (1, [3, 15, 31], 4, True),
    (2, [15, 17, 19, 21, 23, 25, 27, 29], 156, True),
    (3, [33, 62, 63, 64, 65], 16, False),
    (4, [14, 101, 255], 312, True),
    (5, [21], 1, True),
    (6, [15, 29], 500, True),          # 32,000 bins: bins kept in global memory
    (7, [17, 21], 1562, True),         # sketch_size 100,000: 99,968 bins per k
])
def test_sketch_matches_oracle_random(gpu_ctx, seed, kmers, s64, rc):
    from sketchlib_b200 import capi
    rng = np.random.default_rng(seed)
    samples = random_samples(rng, 12, 60_000)
    bases, off, ss = capi.pack_sequences(samples)
    got = capi.sketch(gpu_ctx, bases, off, ss, kmers, s64, use_rc=rc)
    check(got, oracle.sketch(bases, off, ss, kmers, s64, rc))


def test_long_sequences_span_many_work_items(gpu_ctx):
    """Two 1.3 Mb sequences (several 262,144-window items each, N islands on
    item boundaries) and one sample of many reads."""
    from sketchlib_b200 import capi
    rng = np.random.default_rng(11)
    long_a = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 1_300_000)].copy()
    for p in (262_144 - 5, 262_144, 524_288 + 3):
        long_a[p] = ord("N")
    long_b = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 1_300_000)].copy()
    reads = [np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 150)].tobytes() for _ in range(4000)]
    samples = [[long_a.tobytes()], [long_b.tobytes()[:700_000], long_b.tobytes()[700_000:]], reads]
    bases, off, ss = capi.pack_sequences(samples)
    kmers = [15, 21, 31]
    check(capi.sketch(gpu_ctx, bases, off, ss, kmers, 156),
          oracle.sketch(bases, off, ss, kmers, 156, True))


@pytest.mark.parametrize("min_count", [1, 2, 5, 255])
def test_read_filter_matches_oracle(gpu_ctx, min_count):
    from sketchlib_b200 import capi
    rng = np.random.default_rng(min_count)
    genome = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 50_000)]
    samples = []
    for cov in (3, 10):
        reads = []
        for _ in range(cov * 50_000 // 120):
            s = int(rng.integers(0, 50_000 - 120))
            r = genome[s:s + 120].copy()
            err = rng.random(120) < 0.005
            r[err] = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, int(err.sum()))]
            reads.append(r.tobytes())
        samples.append(reads)
    bases, off, ss = capi.pack_sequences(samples)
    kmers = [15, 21, 27]
    check(capi.sketch(gpu_ctx, bases, off, ss, kmers, 64, min_count=min_count),
          oracle.sketch(bases, off, ss, kmers, 64, True, min_count=min_count))


def test_sketch_feeds_the_distance_path(gpu_ctx):
    """GPU sketches give the same distances as the oracle's sketches."""
    from sketchlib_b200 import capi
    rng = np.random.default_rng(21)
    root = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 200_000)]
    samples = []
    for i in range(20):
        g = root.copy()
        m = rng.random(g.size) < 0.002 * i
        g[m] = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, int(m.sum()))]
        samples.append([g.tobytes()])
    bases, off, ss = capi.pack_sequences(samples)
    kmers = list(range(15, 31, 2))
    words, _, _ = capi.sketch(gpu_ctx, bases, off, ss, kmers, 156)
    want, _, _ = oracle.sketch(bases, off, ss, kmers, 156, True)
    np.testing.assert_array_equal(words, want)
    db = capi.Database(gpu_ctx, words, kmers, 156)
    d = capi.dists_dense(gpu_ctx, db)
    db.close()
    np.testing.assert_allclose(d, oracle.dists(want, kmers, 156), atol=1e-6)
    assert d[:19, 0].max() > 0.01 and d[0, 0] < d[18, 0]


def test_sketch_errors(gpu_ctx):
    from sketchlib_b200 import capi
    bases, off, ss = capi.pack_sequences([[b"ACGTACGTACGT"]])
    with pytest.raises(capi.SketchlibError, match="Minimum k must be 3"):
        capi.sketch(gpu_ctx, bases, off, ss, [2, 15], 4)
    with pytest.raises(capi.SketchlibError, match="no sequence"):
        capi.sketch(gpu_ctx, bases, off, np.array([0, 1, 1], np.int64), [15], 4)
    with pytest.raises(capi.SketchlibError, match="min_count"):
        capi.sketch(gpu_ctx, bases, off, ss, [15], 4, min_count=256)
    # the context stays usable
    w, _, dens = capi.sketch(gpu_ctx, bases, off, ss, [5], 4)
    assert dens[0]


@pytest.mark.skipif(not oracle.sketcher_available(), reason="oracle/_ref/libref_sketch.so not built")
def test_64_genomes_match_reference_sketcher(gpu_ctx):
    """The CPU parity case's 64 genomes of 2.5 Mb, sketched on the device and
    by the reference's own sketcher."""
    from sketchlib_b200 import capi
    rs = oracle.RefSketcher()
    genomes = rs.genomes(64, 2_500_000, 0x5EED0001)
    kmers = list(range(15, 31, 2))
    want = rs.sketch(genomes, kmers, 156)
    off = np.arange(65, dtype=np.int64) * 2_500_000
    ss = np.arange(65, dtype=np.int64)
    words, inv, dens = capi.sketch(gpu_ctx, genomes.reshape(-1), off, ss, kmers, 156)
    np.testing.assert_array_equal(words, want)


@pytest.mark.parametrize("min_count,shift", [(0, 0), (0, 3), (2, 5)])
def test_device_entry_point_matches_host_one(gpu_ctx, min_count, shift):
    """sk_sketch_device (device bases, possibly unaligned; device outputs)
    gives sk_sketch's results and leaves the bases unchanged."""
    import torch
    from sketchlib_b200 import capi
    rng = np.random.default_rng(40 + shift)
    samples = random_samples(rng, 9, 200_000)
    bases, off, ss = capi.pack_sequences(samples)
    kmers, s64 = [15, 21, 31], 64
    want = capi.sketch(gpu_ctx, bases, off, ss, kmers, s64, min_count=min_count)
    buf = torch.zeros(bases.size + 16, dtype=torch.uint8, device="cuda")
    buf[shift:shift + bases.size] = torch.from_numpy(bases.copy()).cuda()
    n = len(ss) - 1
    words = torch.empty((n, len(kmers), s64 * 14), dtype=torch.int64, device="cuda")
    inv = torch.empty((n, len(kmers)), dtype=torch.float64, device="cuda")
    dens = torch.empty(n, dtype=torch.uint8, device="cuda")
    capi.sketch_device(gpu_ctx, buf.data_ptr() + shift, off, ss, kmers, s64, words.data_ptr(),
                       min_count=min_count, d_inv_minhash=inv.data_ptr(),
                       d_densified=dens.data_ptr())
    np.testing.assert_array_equal(words.cpu().numpy().view(np.uint64), want[0])
    np.testing.assert_array_equal(inv.cpu().numpy(), want[1])
    np.testing.assert_array_equal(dens.cpu().numpy().astype(bool), want[2])
    np.testing.assert_array_equal(buf[shift:shift + bases.size].cpu().numpy(), bases)


def test_read_filter_in_many_counting_passes():
    """A 1 MiB memory limit shrinks the count table to 256 KB per pass, so a
    read set is counted in about two dozen bin-range passes; the sketch is
    unchanged."""
    from sketchlib_b200 import capi
    rng = np.random.default_rng(77)
    genome = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 50_000)]
    reads = []
    for _ in range(3 * 50_000 // 100):
        s = int(rng.integers(0, 50_000 - 100))
        r = genome[s:s + 100].copy()
        e = rng.random(100) < 0.01
        r[e] = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, int(e.sum()))]
        reads.append(r.tobytes())
    bases, off, ss = capi.pack_sequences([reads])
    kmers = [15, 21, 27]
    with capi.Context(0) as ctx:
        ctx.set_memory_limit(1 << 20)
        got = capi.sketch(ctx, bases, off, ss, kmers, 64, min_count=2)
    check(got, oracle.sketch(bases, off, ss, kmers, 64, True, min_count=2))


def test_many_samples_split_into_batches(gpu_ctx):
    """300 samples at 64,000 bins and 8 k-mer lengths: 1.2 GB of bins rows,
    more than one batch holds, and bins too large for shared memory."""
    from sketchlib_b200 import capi
    rng = np.random.default_rng(78)
    samples = [[np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 100_000)].tobytes()]
               for _ in range(300)]
    bases, off, ss = capi.pack_sequences(samples)
    kmers = list(range(15, 31, 2))
    check(capi.sketch(gpu_ctx, bases, off, ss, kmers, 1000),
          oracle.sketch(bases, off, ss, kmers, 1000, True))


@pytest.mark.parametrize("seed,kmers,s64,rc,min_count", [
    (31, [3, 15, 17], 16, True, 0),
    (32, [9, 21, 29], 156, False, 0),
    (33, [15, 85, 255], 64, True, 0),     # windows of 253, 763 bases
    (34, [15, 21], 64, True, 2),          # read filter with spaced seeds
])
def test_codon_phased_matches_oracle(gpu_ctx, seed, kmers, s64, rc, min_count):
    from sketchlib_b200 import capi
    rng = np.random.default_rng(seed)
    if min_count:
        genome = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 30_000)]
        reads = []
        for _ in range(4 * 30_000 // 150):
            s = int(rng.integers(0, 30_000 - 150))
            reads.append(genome[s:s + 150].tobytes())
        samples = [reads]
    else:
        samples = random_samples(rng, 8, 80_000)
    bases, off, ss = capi.pack_sequences(samples)
    got = capi.sketch(gpu_ctx, bases, off, ss, kmers, s64, use_rc=rc, min_count=min_count,
                      codon_phased=True)
    check(got, oracle.sketch(bases, off, ss, kmers, s64, rc, min_count=min_count,
                             codon_phased=True))


def test_codon_phased_device_entry_point(gpu_ctx):
    import torch
    from sketchlib_b200 import capi
    rng = np.random.default_rng(35)
    bases, off, ss = capi.pack_sequences(random_samples(rng, 5, 100_000))
    kmers = [15, 21]
    want = capi.sketch(gpu_ctx, bases, off, ss, kmers, 64, codon_phased=True)
    buf = torch.from_numpy(bases.copy()).cuda()
    words = torch.empty((5, 2, 64 * 14), dtype=torch.int64, device="cuda")
    capi.sketch_device(gpu_ctx, buf.data_ptr(), off, ss, kmers, 64, words.data_ptr(),
                       codon_phased=True)
    np.testing.assert_array_equal(words.cpu().numpy().view(np.uint64), want[0])


@pytest.mark.parametrize("min_count", [2, 40])
def test_read_filter_with_skewed_hash_groups(gpu_ctx, min_count):
    """Counting groups hashes by range of their sign; low-complexity reads
    (homopolymers, short tandem repeats, thousands of copies of one read) pile
    most occurrences into a few groups, next to ordinary reads spread over all
    of them.  The sketch equals the oracle's exact count."""
    from sketchlib_b200 import capi
    rng = np.random.default_rng(91 + min_count)
    genome = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, 40_000)]
    reads = []
    for _ in range(6 * 40_000 // 100):
        s = int(rng.integers(0, 40_000 - 100))
        r = genome[s:s + 100].copy()
        e = rng.random(100) < 0.01
        r[e] = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, int(e.sum()))]
        reads.append(r.tobytes())
    copy = genome[1000:1100].tobytes()
    reads += [b"A" * 100, b"CA" * 50, b"GGT" * 33 + b"G"] * 300 + [copy] * 3000
    order = rng.permutation(len(reads))
    bases, off, ss = capi.pack_sequences([[reads[i] for i in order]])
    kmers = [15, 21, 27]
    check(capi.sketch(gpu_ctx, bases, off, ss, kmers, 64, min_count=min_count),
          oracle.sketch(bases, off, ss, kmers, 64, True, min_count=min_count))
