"""Golden vectors of the reference's sketcher, for the sketching parity tests.

Runs pp-sketchlib's own CPU sketch() (src/sketch/sketch.cpp:120-168, compiled
from the reference sources into oracle/_ref/libref_sketch.so by
oracle/Makefile) on seeded inputs and stores inputs and outputs in
tests/golden/sketch_golden.npz, so the tests need neither the reference tree
nor its build:

  seqs_*     assemblies-like samples given as sequences (sk_sketch's flat form:
             bases, seq_off, sample_seqs) covering several sequences per
             sample, N runs, lower case, U, IUPAC letters, sequences shorter
             than k, an all-N sample and a sample of one k-mer;
             sketched for five (kmers, sketchsize64, use_rc, codon_phased)
             settings through SeqBuf(std::vector<std::string>) -- sequences as
             given; the last two use the codon-phased spaced seeds.
  reads_*    a read set (FASTQ with N-containing and short reads) sketched
             through SeqBuf(files, largest k) with min_count = 2 and 3 and the
             exact counter (`exact = true`); the fixture keeps the reads as
             written, the tests apply SeqBuf's rules (upper case, reads
             shorter than the largest k dropped).

Usage: python tests/golden/make_sketch_golden.py   (after `make -f oracle/Makefile`)
"""
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
import oracle  # noqa: E402

rng = np.random.default_rng(0x5EED5E)


def rseq(n, p_n=0.0, alphabet=b"ACGT"):
    a = np.frombuffer(alphabet, np.uint8)[rng.integers(0, len(alphabet), n)].copy()
    if p_n:
        a[rng.random(n) < p_n] = ord("N")
    return a.tobytes()


genome = rseq(6000)
samples = [
    [rseq(3000)],
    [rseq(500), rseq(40), rseq(1200, 0.01), b"", rseq(2)],
    [rseq(2000, alphabet=b"acgtACGTUuNRYKMacgt")],
    [b"NNNNNNNNNNNNNNNNNNNN"],
    [rseq(10)],
    [rseq(20000, 0.001)],
    [genome[i:i + 100] for i in range(0, 5900, 37)],
    [b"ACGT" * 300],
    [rseq(15)],
    [genome[:3000], genome[2500:6000].lower()],
]
bases, seq_off, sample_seqs = oracle.pack_samples(samples)
settings = [([3, 15, 31, 33], 4, True, False), ([15, 17, 63, 64, 101], 4, False, False),
            ([21, 29], 156, True, False), ([3, 9, 15], 4, True, True), ([5, 11, 17], 16, False, True)]
rs = oracle.RefSketcher()
out = {"seqs_bases": bases, "seqs_seq_off": seq_off, "seqs_sample_seqs": sample_seqs}
for i, (kmers, s64, rc, phased) in enumerate(settings):
    words, inv, dens = rs.sketch_seqs(bases, seq_off, sample_seqs, kmers, s64, rc,
                                      codon_phased=phased)
    out[f"seqs{i}_kmers"] = np.asarray(kmers, np.int32)
    out[f"seqs{i}_s64"] = np.int32(s64)
    out[f"seqs{i}_use_rc"] = np.int32(rc)
    out[f"seqs{i}_codon_phased"] = np.int32(phased)
    out[f"seqs{i}_words"] = words
    out[f"seqs{i}_inv_minhash"] = inv
    out[f"seqs{i}_densified"] = dens

# read set: 8x coverage of a 20 kb genome, 1% substitutions, some Ns and short reads
ref_genome = np.frombuffer(rseq(20000), np.uint8)
reads = []
for _ in range(1600):
    start = int(rng.integers(0, 20000 - 100))
    length = int(rng.choice([100, 100, 100, 30, 12]))
    r = ref_genome[start:start + length].copy()
    err = rng.random(length) < 0.01
    r[err] = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, int(err.sum()))]
    if rng.random() < 0.05:
        r[int(rng.integers(0, length))] = ord("N")
    q = r.tobytes()
    reads.append(q.lower() if rng.random() < 0.3 else q)
read_kmers = [15, 21]
with tempfile.TemporaryDirectory() as tmp:
    fq = Path(tmp) / "reads.fastq"
    with open(fq, "wb") as f:
        for i, r in enumerate(reads):
            f.write(b"@r%d\n%s\n+\n%s\n" % (i, r, b"I" * len(r)))
    for mc in (2, 3):
        words, inv, dens, is_reads = rs.sketch_file(fq, read_kmers, 16, True, mc, True)
        assert is_reads
        out[f"reads_mc{mc}_words"] = words
        out[f"reads_mc{mc}_inv_minhash"] = inv
        out[f"reads_mc{mc}_densified"] = np.bool_(dens)
r_bases, r_off, _ = oracle.pack_samples([reads])
out["reads_bases"] = r_bases
out["reads_seq_off"] = r_off
out["reads_kmers"] = np.asarray(read_kmers, np.int32)
out["reads_s64"] = np.int32(16)

dest = Path(__file__).with_name("sketch_golden.npz")
np.savez_compressed(dest, **out)
print(f"wrote {dest} ({dest.stat().st_size} bytes)")
