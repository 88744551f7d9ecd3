"""constructDatabase end to end on the GPU: sequence files in, an HDF5 sketch
database out, against the reference's own file reader and sketcher
(SeqBuf + sketch(), oracle/_ref/libref_sketch.so), then queryDatabase on the
new database against the oracle."""
import gzip

import numpy as np
import pytest

import oracle

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.sketcher_available(),
                                 reason="oracle/_ref/libref_sketch.so not built")]

KMERS = [15, 19, 23, 27]
S64 = 64


def genomes(rng, n, length):
    root = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, length)]
    out = []
    for i in range(n):
        g = root.copy()
        m = rng.random(length) < 0.004 * i
        g[m] = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, int(m.sum()))]
        out.append(g)
    return out


def write_fasta(path, g, rng):
    cuts = sorted(rng.integers(1, len(g) - 1, 3).tolist())
    parts, prev = [], 0
    for i, c in enumerate(cuts + [len(g)]):
        s = g[prev:c].tobytes()
        parts.append(b">c%d\n" % i + b"\n".join(s[j:j + 80] for j in range(0, len(s), 80)) + b"\n")
        prev = c
    text = b"".join(parts).replace(b"ACGTA", b"ACGNA", 3)
    path.write_bytes(gzip.compress(text) if path.suffix == ".gz" else text)


def write_fastq(path, g, rng, cover=8, read_len=100):
    parts = []
    for i in range(cover * len(g) // read_len):
        s = int(rng.integers(0, len(g) - read_len))
        r = g[s:s + read_len].copy()
        e = rng.random(read_len) < 0.01
        r[e] = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, int(e.sum()))]
        parts.append(b"@r%d\n%s\n+\n%s\n" % (i, r.tobytes(), b"I" * read_len))
    path.write_bytes(b"".join(parts))


def test_construct_database_matches_reference_sketcher(tmp_path):
    import pp_sketchlib
    rng = np.random.default_rng(3)
    gs = genomes(rng, 5, 200_000)
    names, files = [], []
    for i, g in enumerate(gs):
        p = tmp_path / (f"asm{i}.fa.gz" if i % 2 else f"asm{i}.fa")
        write_fasta(p, g, rng)
        names.append(f"asm{i}")
        files.append([str(p)])
    for i, g in enumerate(genomes(rng, 2, 50_000)):
        p = tmp_path / f"reads{i}.fq"
        write_fastq(p, g, rng)
        names.append(f"reads{i}")
        files.append([str(p)])
    db = str(tmp_path / "db")
    pp_sketchlib.constructDatabase(db, names, files, KMERS, S64, calc_random=False,
                                   min_count=2, exact=True, num_threads=4)
    got = pp_sketchlib._load_sketch_db(db, names=names, klist=KMERS)
    rs = oracle.RefSketcher()
    for i, (name, f) in enumerate(zip(names, files)):
        words, inv, _, is_reads = rs.sketch_file(f[0], KMERS, S64, True, 2, True)
        np.testing.assert_array_equal(got["words"][i], words, err_msg=name)
        info = rs.seqbuf(f[0], KMERS[-1])
        want_len = int(len(KMERS) / inv.sum()) if is_reads else info["total"]
        assert got["length"][i] == want_len, name
        np.testing.assert_array_equal(got["base_freq"][i], info["base_freq"])

    # distances on the new database
    d = pp_sketchlib.queryDatabase(db, db, names, names, KMERS, random_correct=False)
    np.testing.assert_allclose(d, oracle.dists(got["words"], KMERS, S64), atol=1e-6)

    # an existing database holding every sample is kept as it is
    before = (tmp_path / "db.h5").read_bytes()
    pp_sketchlib.constructDatabase(db, names, files, KMERS, S64, calc_random=False)
    assert (tmp_path / "db.h5").read_bytes() == before


def test_construct_database_codon_phased(tmp_path):
    """codon_phased=True sketches with the reference's spaced seeds (the
    reference's CPU sketcher does; its GPU sketcher refuses)."""
    import pp_sketchlib
    rng = np.random.default_rng(4)
    names, files = [], []
    for i, g in enumerate(genomes(rng, 3, 100_000)):
        p = tmp_path / f"g{i}.fa"
        write_fasta(p, g, rng)
        names.append(f"g{i}")
        files.append([str(p)])
    db = str(tmp_path / "phased")
    kmers = [15, 19]
    pp_sketchlib.constructDatabase(db, names, files, kmers, S64, codon_phased=True,
                                   calc_random=False)
    got = pp_sketchlib._load_sketch_db(db, names=names, klist=kmers)
    rs = oracle.RefSketcher()
    for i, f in enumerate(files):
        info = rs.seqbuf(f[0], kmers[-1])
        bases, off, ss = oracle.pack_samples([[q.encode() for q in info["seqs"]]])
        want = rs.sketch_seqs(bases, off, ss, kmers, S64, True, codon_phased=True)[0]
        np.testing.assert_array_equal(got["words"][i], want[0])


def test_construct_database_errors(tmp_path):
    import pp_sketchlib
    empty = tmp_path / "empty.fa"
    empty.write_bytes(b">x\nACGT\n")          # shorter than the largest k: nothing kept
    with pytest.raises(RuntimeError, match="contains no sequence"):
        pp_sketchlib.constructDatabase(str(tmp_path / "e"), ["e"], [[str(empty)]], KMERS, S64)
    with pytest.raises(RuntimeError, match="cannot name a database group"):
        pp_sketchlib.constructDatabase(str(tmp_path / "s"), ["a/b"], [[str(empty)]], KMERS, S64)
