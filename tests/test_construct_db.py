"""constructDatabase's host parts on the CPU: the HDF5 database writer (round
trip through this library's reader, plus the file-format invariants that
libhdf5 relies on, checked by an independent walker below) and the
FASTA/FASTQ reader against the reference's own SeqBuf
(src/sketch/seqio.cpp:55-100, compiled into oracle/_ref/libref_sketch.so)."""
import gzip
import struct

import numpy as np
import pytest

import oracle


def pp():
    import pp_sketchlib
    return pp_sketchlib


# ------------------------------------------------------------ HDF5 writer

def walk_h5(path):
    """Walks a written file by the HDF5 format specification (superblock v0,
    v1 object headers, symbol-table groups) and checks its invariants;
    returns {group path: sorted member names}."""
    d = open(path, "rb").read()
    assert d[:8] == b"\x89HDF\r\n\x1a\n"
    assert list(d[8:16]) == [0, 0, 0, 0, 0, 8, 8, 0]
    assert struct.unpack("<HHI", d[16:24]) == (4, 16, 0)
    base, free, eof, drv = struct.unpack("<QQQQ", d[24:56])
    assert (base, free, drv) == (0, 2**64 - 1, 2**64 - 1) and eof == len(d)
    name_off, root, cache = struct.unpack("<QQI", d[56:76])
    assert name_off == 0 and cache == 1
    groups = {}

    def header(addr):
        v, _, nmsg, rc, size = struct.unpack("<BBHII", d[addr:addr + 12])
        assert v == 1 and rc == 1 and addr % 8 == 0
        msgs, p = [], addr + 16
        while p < addr + 16 + size:
            t, sz, fl = struct.unpack("<HHB", d[p:p + 5])
            assert sz % 8 == 0
            msgs.append((t, d[p + 8:p + 8 + sz]))
            p += 8 + sz
        assert p == addr + 16 + size and len(msgs) == nmsg
        return msgs

    def heap_name(heap, off):
        assert d[heap:heap + 4] == b"HEAP"
        seg, free_at, data = struct.unpack("<QQQ", d[heap + 8:heap + 32])
        assert off < seg and free_at < seg
        assert struct.unpack("<Q", d[data + free_at:data + free_at + 8])[0] == 1   # no next free block
        return d[data + off:d.index(b"\0", data + off)].decode()

    def btree(addr, heap, level_expected=None):
        assert d[addr:addr + 4] == b"TREE" and d[addr + 4] == 0
        level, n = d[addr + 5], struct.unpack("<H", d[addr + 6:addr + 8])[0]
        assert n <= 32
        vals = struct.unpack("<" + "Q" * (2 * n + 1), d[addr + 24:addr + 24 + 8 * (2 * n + 1)])
        keys, kids = vals[0::2], vals[1::2]
        names = [heap_name(heap, k) for k in keys]
        assert names == sorted(names)
        out = []
        for i, c in enumerate(kids):
            got = btree(c, heap) if level > 0 else snod(c, heap)
            assert got and names[i] < got[0][0] or (i == 0 and names[0] == "")
            assert got[-1][0] == names[i + 1]
            out += got
        return out

    def snod(addr, heap):
        assert d[addr:addr + 4] == b"SNOD" and d[addr + 4] == 1
        n = struct.unpack("<H", d[addr + 6:addr + 8])[0]
        assert 1 <= n <= 8
        ents = []
        for i in range(n):
            e = addr + 8 + 40 * i
            off, hdr, cache = struct.unpack("<QQI", d[e:e + 20])
            scratch = struct.unpack("<QQ", d[e + 24:e + 40])
            ents.append((heap_name(heap, off), hdr, cache, scratch))
        assert [x[0] for x in ents] == sorted(x[0] for x in ents)
        return ents

    def group(path_, addr, cached=None):
        msgs = header(addr)
        assert msgs[0][0] == 0x11
        bt, hp = struct.unpack("<QQ", msgs[0][1][:16])
        if cached is not None:
            assert cached == (bt, hp)
        members = btree(bt, hp)
        groups[path_] = [m[0] for m in members]
        for name, hdr, cache, scratch in members:
            sub = header(hdr)
            if sub[0][0] == 0x11:
                assert cache == 1
                group(path_.rstrip("/") + "/" + name, hdr, scratch)
            else:
                assert cache == 0
                types = [t for t, _ in sub]
                assert types[:4] == [0x0001, 0x0003, 0x0005, 0x0008]
                layout = sub[3][1]
                assert layout[0] == 3 and layout[1] == 1
                a, size = struct.unpack("<QQ", layout[2:18])
                assert a + size <= len(d)

    group("/", root, struct.unpack("<QQ", d[80:96]))
    return groups


@pytest.mark.parametrize("n", [1, 9, 600])
def test_h5_writer_round_trip(tmp_path, n):
    rng = np.random.default_rng(n)
    kmers, s64 = [15, 17, 21], 4
    words = rng.integers(0, 2 ** 64, size=(n, len(kmers), s64 * 14), dtype=np.uint64)
    names = [f"sample_{i:04d}" for i in rng.permutation(n)]
    lengths = list(range(1000, 1000 + n))
    db = str(tmp_path / "db")
    pp()._save_sketch_db(db, names, words, kmers, s64, lengths=lengths)
    got = pp()._load_sketch_db(db, names=names, klist=kmers)
    np.testing.assert_array_equal(got["words"], words)
    assert list(got["names"]) == names and list(got["length"]) == lengths
    groups = walk_h5(db + ".h5")
    assert groups["/"] == ["sketches"]
    assert groups["/sketches"] == sorted(names)
    assert groups["/sketches/" + names[0]] == sorted(str(k) for k in kmers)


# ------------------------------------------------------- FASTA/FASTQ reader

needs_ref = pytest.mark.skipif(not oracle.sketcher_available(),
                               reason="oracle/_ref/libref_sketch.so not built")


def rseq(rng, n, alphabet=b"ACGT"):
    return np.frombuffer(alphabet, np.uint8)[rng.integers(0, len(alphabet), n)].tobytes()


def fasta_text(rng):
    parts = []
    for i in range(12):
        s = rseq(rng, int(rng.integers(0, 3000)), b"ACGTacgtNNRU")
        parts.append(b">contig%d some comment\n" % i)
        width = int(rng.choice([60, 80, 1000]))
        for j in range(0, len(s), width):
            parts.append(s[j:j + width] + (b"\r\n" if i % 3 == 0 else b"\n"))
        if i % 4 == 1:
            parts.append(b"\n")   # an empty line
    parts.append(b">tail_no_newline\n" + rseq(rng, 50))
    return b"".join(parts)


def fastq_text(rng):
    parts = []
    for i in range(400):
        s = rseq(rng, int(rng.choice([100, 150, 20])), b"ACGTN")
        q = bytes(rng.integers(33, 75, len(s)).astype(np.uint8))
        if i % 50 == 7:
            q = b"@" + q[1:]          # a quality line starting with '@'
        parts.append(b"@read%d\n%s\n+read%d\n%s\n" % (i, s, i, q))
    return b"".join(parts)


@needs_ref
@pytest.mark.parametrize("kind", ["fasta", "fasta.gz", "fastq", "fastq.gz"])
def test_read_sequences_matches_reference_seqbuf(tmp_path, kind):
    rng = np.random.default_rng(len(kind))
    text = fastq_text(rng) if kind.startswith("fastq") else fasta_text(rng)
    path = tmp_path / f"in.{kind}"
    path.write_bytes(gzip.compress(text) if kind.endswith(".gz") else text)
    want = oracle.RefSketcher().seqbuf(path, 31)
    got = pp()._read_sequences([str(path)], 31)
    assert got["seqs"] == want["seqs"]
    for key in ("total", "missing_bases", "reads", "max_length"):
        assert got[key] == want[key], key
    np.testing.assert_array_equal(got["base_freq"], want["base_freq"])


def test_read_sequences_errors(tmp_path):
    with pytest.raises(RuntimeError, match="Could not open"):
        pp()._read_sequences([str(tmp_path / "missing.fa")], 15)
