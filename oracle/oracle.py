"""ctypes wrapper of the CPU oracle (sk_oracle.c) and of the reference
harness built from the reference sources (_ref/libref_querydb.so, the
reference sketcher _ref/libref_sketch.so and GPU kernel _ref/libref_gpu.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / --impl reference legs of bench.py, as the checker and the CPU
baseline.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
REF_PATH = HERE / "_ref" / "libref_querydb.so"


class _Random(C.Structure):
    _fields_ = [("mode", C.c_int), ("use_rc", C.c_int), ("n_clusters", C.c_int),
                ("table", C.c_void_p), ("cl_rows", C.c_void_p), ("cl_cols", C.c_void_p),
                ("len_rows", C.c_void_p), ("len_cols", C.c_void_p)]


def build():
    """Compiles the oracle (and the reference harness where the reference
    sources are present) with oracle/Makefile."""
    import subprocess
    subprocess.run(["make", "-s", "-f", str(HERE / "Makefile")], check=True)


def _load():
    if not LIB_PATH.exists():
        build()
    lib = C.CDLL(str(LIB_PATH))
    vp, i32, i64 = C.c_void_p, C.c_int, C.c_int64
    lib.sko_intersize.restype = C.c_uint32
    lib.sko_intersize.argtypes = [vp, vp, i32, i32]
    lib.sko_csrs.restype = C.c_double
    lib.sko_csrs.argtypes = [i32, i32, C.c_uint64, C.c_uint64]
    lib.sko_jaccard.restype = C.c_double
    lib.sko_jaccard.argtypes = [C.c_uint32, i32, C.c_double]
    for f in (lib.sko_fit_slope_f64, lib.sko_fit_slope_f32):
        f.restype = None
        f.argtypes = [vp, vp, i32, i32, vp, vp]
    lib.sko_dists.restype = None
    lib.sko_dists.argtypes = [vp, i64, vp, i64, i32, i32, vp, i32, i32, C.POINTER(_Random), i32,
                              i32, vp, i32]
    lib.sko_dists_multi.restype = i64
    lib.sko_dists_multi.argtypes = [vp, i64, vp, i64, i32, i32, vp, i32, i32, C.POINTER(_Random),
                                    i64, i64, vp, vp, vp, i32]
    lib.sko_dists_self_rows.restype = i64
    lib.sko_dists_self_rows.argtypes = [vp, i64, i32, vp, i32, i32, i64, i64, vp, i32]
    lib.sko_knn_self.restype = None
    lib.sko_knn_self.argtypes = [vp, i64, i32, i32, i32, i32, vp, vp, vp]
    lib.sko_sparsify.restype = i64
    lib.sko_sparsify.argtypes = [vp, i64, i32, i32, C.c_float, vp, vp, vp]
    lib.sko_long_to_square.restype = None
    lib.sko_long_to_square.argtypes = [vp, i64, vp, vp, i64, vp]
    lib.sko_square_to_long.restype = None
    lib.sko_square_to_long.argtypes = [vp, i64, vp]
    lib.sko_closest_cluster.restype = None
    lib.sko_closest_cluster.argtypes = [vp, i32, i32, vp, i64, vp]
    lib.sko_synth_words.restype = i32
    lib.sko_synth_words.argtypes = [vp, vp, i64, i32, i32, C.c_uint64, vp, i32]
    lib.sko_sketch_samples.restype = None
    lib.sko_sketch_samples.argtypes = [vp, vp, vp, i64, vp, i32, i32, i32, i32, i32, i32, vp, vp,
                                       vp, i32]
    return lib


lib = _load()
NTHREADS = os.cpu_count() or 1


def _p(a):
    return None if a is None else a.ctypes.data


class RandomSpec:
    """mode 0 none, 1 equal base (per-sample lengths), 2 table [K][C][C] + clusters."""

    def __init__(self, mode=0, use_rc=True, table=None, cl_rows=None, cl_cols=None,
                 len_rows=None, len_cols=None):
        self.mode = mode
        self.use_rc = use_rc
        self.table = None if table is None else np.ascontiguousarray(table, np.float32)
        self.cl_rows = None if cl_rows is None else np.ascontiguousarray(cl_rows, np.uint16)
        self.cl_cols = None if cl_cols is None else np.ascontiguousarray(cl_cols, np.uint16)
        self.len_rows = None if len_rows is None else np.ascontiguousarray(len_rows, np.uint64)
        self.len_cols = None if len_cols is None else np.ascontiguousarray(len_cols, np.uint64)

    def struct(self):
        return _Random(self.mode, int(self.use_rc),
                       0 if self.table is None else self.table.shape[-1],
                       _p(self.table), _p(self.cl_rows), _p(self.cl_cols), _p(self.len_rows),
                       _p(self.len_cols))


def dists(ref_words, kmers, s64, query_words=None, random: RandomSpec | None = None,
          out_mode=0, regress=0, threads=NTHREADS, bbits=14):
    """Dense distances (self when query_words is None), reference long-form order."""
    cols = np.ascontiguousarray(ref_words, dtype=np.uint64)
    self_ = query_words is None
    rows = cols if self_ else np.ascontiguousarray(query_words, dtype=np.uint64)
    n_cols, n_rows = cols.shape[0], rows.shape[0]
    K = len(kmers)
    km = np.ascontiguousarray(kmers, dtype=np.int32)
    pairs = n_cols * (n_cols - 1) // 2 if self_ else n_rows * n_cols
    if out_mode == 0:
        out = np.zeros((pairs, 2), np.float32)
    elif out_mode == 1:
        out = np.zeros((pairs, K), np.float32)
    else:
        out = np.zeros((pairs, K), np.uint32)
    rs = (random or RandomSpec()).struct()
    lib.sko_dists(rows.ctypes.data, n_rows, cols.ctypes.data, n_cols, int(self_), K,
                  km.ctypes.data, s64, bbits, C.byref(rs), out_mode, regress, out.ctypes.data,
                  threads)
    return out


def dists_multi(ref_words, kmers, s64, query_words=None, random: RandomSpec | None = None,
                row_begin=0, row_end=None, threads=NTHREADS, bbits=14):
    """Jaccard (pairs, K), double fit and float-LDLT fit (pairs, 2) of rows
    [row_begin, row_end) from one intersection pass, long-form order."""
    cols = np.ascontiguousarray(ref_words, dtype=np.uint64)
    self_ = query_words is None
    rows = cols if self_ else np.ascontiguousarray(query_words, dtype=np.uint64)
    n_cols, n_rows = cols.shape[0], rows.shape[0]
    outer = n_cols if self_ else n_rows
    row_end = outer if row_end is None else row_end
    K = len(kmers)
    km = np.ascontiguousarray(kmers, dtype=np.int32)
    if self_:
        def first(i):
            return n_cols * i - i * (i + 1) // 2
        pairs = first(row_end) - first(row_begin)
    else:
        pairs = (row_end - row_begin) * n_cols
    jac = np.zeros((pairs, K), np.float32)
    f64 = np.zeros((pairs, 2), np.float32)
    f32 = np.zeros((pairs, 2), np.float32)
    rs = (random or RandomSpec()).struct()
    done = lib.sko_dists_multi(rows.ctypes.data, n_rows, cols.ctypes.data, n_cols, int(self_), K,
                               km.ctypes.data, s64, bbits, C.byref(rs), row_begin, row_end,
                               jac.ctypes.data, f64.ctypes.data, f32.ctypes.data, threads)
    assert done == pairs
    return jac, f64, f32


def dists_self_rows(words, kmers, s64, row_begin, row_end, out, threads=NTHREADS, bbits=14):
    """Core/accessory of all-vs-all rows [row_begin, row_end) into the full
    long-form `out`; returns the number of pairs computed."""
    w = np.ascontiguousarray(words, np.uint64)
    km = np.ascontiguousarray(kmers, np.int32)
    return lib.sko_dists_self_rows(w.ctypes.data, w.shape[0], len(km), km.ctypes.data, s64, bbits,
                                   row_begin, row_end, out.ctypes.data, threads)


def closest_cluster(centroids, base_freq, use_rc=True):
    """Cluster ids [n] of compositions base_freq [n][4] against centroids [C][4]."""
    c = np.ascontiguousarray(centroids, np.float32)
    b = np.ascontiguousarray(base_freq, np.float64).reshape(-1, 4)
    out = np.zeros(b.shape[0], np.uint16)
    lib.sko_closest_cluster(c.ctypes.data, c.shape[0], int(use_rc), b.ctypes.data, b.shape[0],
                            out.ctypes.data)
    return out


def synth_words(parent, thresh, s64, seed, threads=NTHREADS):
    """Reference-layout words [n][K][s64 * 14] of the seeded bin-level tree
    generator (parent / thresh from synth.random_tree and friends), computed
    here so a caller needs nothing from the library under test."""
    parent = np.ascontiguousarray(parent, np.int32)
    thresh = np.ascontiguousarray(thresh, np.uint32)
    n, K = thresh.shape
    words = np.empty((n, K, s64 * 14), np.uint64)
    rc = lib.sko_synth_words(parent.ctypes.data, thresh.ctypes.data, n, K, s64,
                             C.c_uint64(seed & (2 ** 64 - 1)), words.ctypes.data, threads)
    if rc != 0:
        raise ValueError("parents must precede their children")
    return words


def intersize(a, b, s64, bbits=14):
    a = np.ascontiguousarray(a, np.uint64)
    b = np.ascontiguousarray(b, np.uint64)
    return lib.sko_intersize(a.ctypes.data, b.ctypes.data, s64, bbits)


def csrs(k, use_rc, l1, l2):
    return lib.sko_csrs(k, int(use_rc), l1, l2)


def jaccard(intersize_, s64, random_jaccard=0.0):
    return lib.sko_jaccard(intersize_, s64, random_jaccard)


def fit_slope(J, kmers, s64, f32=False):
    J = np.ascontiguousarray(J, np.float32)
    km = np.ascontiguousarray(kmers, np.int32)
    core, acc = C.c_float(), C.c_float()
    fn = lib.sko_fit_slope_f32 if f32 else lib.sko_fit_slope_f64
    fn(J.ctypes.data, km.ctypes.data, len(km), s64, C.byref(core), C.byref(acc))
    return core.value, acc.value


def knn_self(long_form, n, col, kNN, jaccard_=False):
    lf = np.ascontiguousarray(long_form, np.float32)
    if lf.ndim == 1:
        lf = lf.reshape(-1, 1)
    i = np.empty(n * kNN, np.int64)
    j = np.empty(n * kNN, np.int64)
    d = np.empty(n * kNN, np.float32)
    lib.sko_knn_self(lf.ctypes.data, n, lf.shape[1], col, int(jaccard_), kNN, i.ctypes.data,
                     j.ctypes.data, d.ctypes.data)
    return i, j, d


def sparsify(long_form, n, col, cutoff):
    lf = np.ascontiguousarray(long_form, np.float32)
    if lf.ndim == 1:
        lf = lf.reshape(-1, 1)
    m = lib.sko_sparsify(lf.ctypes.data, n, lf.shape[1], col, cutoff, None, None, None)
    i = np.empty(m, np.int64)
    j = np.empty(m, np.int64)
    d = np.empty(m, np.float32)
    lib.sko_sparsify(lf.ctypes.data, n, lf.shape[1], col, cutoff, i.ctypes.data, j.ctypes.data,
                     d.ctypes.data)
    return i, j, d


def long_to_square(rr, n_rr, qr=None, qq=None, n_qq=0):
    rr = np.ascontiguousarray(rr, np.float32)
    qr = None if qr is None else np.ascontiguousarray(qr, np.float32)
    qq = None if qq is None else np.ascontiguousarray(qq, np.float32)
    n = n_rr + n_qq
    out = np.zeros((n, n), np.float32)
    lib.sko_long_to_square(rr.ctypes.data, n_rr, _p(qr), _p(qq), n_qq, out.ctypes.data)
    return out


def square_to_long(sq):
    sq = np.ascontiguousarray(sq, np.float32)
    n = sq.shape[0]
    out = np.zeros(n * (n - 1) // 2, np.float32)
    lib.sko_square_to_long(sq.ctypes.data, n, out.ctypes.data)
    return out


# ----------------------------------------------------- reference harness

class RefQueryDb:
    """query_db's all-vs-all loop around the reference's compiled
    calc_intersize (oracle/_ref).  Available when it was built."""

    def __init__(self):
        if not REF_PATH.exists():
            raise FileNotFoundError(f"{REF_PATH} not built (needs the reference sources)")
        lib_ = C.CDLL(str(REF_PATH))
        vp, i32, i64 = C.c_void_p, C.c_int, C.c_int64
        lib_.ref_sketches_create.restype = vp
        lib_.ref_sketches_create.argtypes = [vp, i64, i32, i32, i32]
        lib_.ref_sketches_destroy.restype = None
        lib_.ref_sketches_destroy.argtypes = [vp]
        lib_.ref_query_db_self.restype = i64
        lib_.ref_query_db_self.argtypes = [vp, i64, i32, vp, i32, i32, i64, i64, vp, i32]
        lib_.ref_intersize.restype = C.c_uint32
        lib_.ref_intersize.argtypes = [vp, vp, i32, i32]
        self.lib = lib_

    def intersize(self, a, b, s64, bbits=14):
        a = np.ascontiguousarray(a, np.uint64)
        b = np.ascontiguousarray(b, np.uint64)
        return self.lib.ref_intersize(a.ctypes.data, b.ctypes.data, s64, bbits)

    def prepare(self, words, kmers, s64, bbits=14):
        """Holds the sketches as per-sample, per-k std::vector<uint64_t>."""
        w = np.ascontiguousarray(words, np.uint64)
        return (self.lib.ref_sketches_create(w.ctypes.data, w.shape[0], len(kmers), s64, bbits),
                w.shape[0], np.ascontiguousarray(kmers, np.int32), s64, bbits)

    def release(self, prepared):
        self.lib.ref_sketches_destroy(prepared[0])

    def run_rows(self, prepared, row_begin, row_end, out, threads=NTHREADS):
        h, n, km, s64, bbits = prepared
        return self.lib.ref_query_db_self(h, n, len(km), km.ctypes.data, s64, bbits, row_begin,
                                          row_end, out.ctypes.data, threads)

    def self_dists(self, words, kmers, s64, row_begin=0, row_end=None, threads=NTHREADS,
                   bbits=14, out=None):
        n = np.asarray(words).shape[0]
        if out is None:
            out = np.zeros((n * (n - 1) // 2, 2), np.float32)
        prep = self.prepare(words, kmers, s64, bbits)
        try:
            done = self.run_rows(prep, row_begin, n if row_end is None else row_end, out, threads)
        finally:
            self.release(prep)
        return out, done


def pack_samples(samples):
    """Samples given as lists of sequences (str or bytes) -> (bases uint8,
    seq_off int64 [n_seqs + 1], sample_seqs int64 [n + 1])."""
    seqs = [q.encode() if isinstance(q, str) else bytes(q) for smp in samples for q in smp]
    lens = np.array([len(q) for q in seqs], np.int64)
    seq_off = np.zeros(len(seqs) + 1, np.int64)
    np.cumsum(lens, out=seq_off[1:])
    counts = np.array([len(smp) for smp in samples], np.int64)
    sample_seqs = np.zeros(len(samples) + 1, np.int64)
    np.cumsum(counts, out=sample_seqs[1:])
    bases = np.frombuffer(b"".join(seqs), np.uint8).copy() if seqs else np.zeros(0, np.uint8)
    return bases, seq_off, sample_seqs


def sketch(bases, seq_off, sample_seqs, kmers, s64, use_rc=True, min_count=0, threads=NTHREADS,
           bbits=14, codon_phased=False):
    """The oracle's sketcher (sko_sketch_samples): words [n][K][s64*bbits],
    inv_minhash [n][K], densified [n]; min_count > 0 keeps hashes seen that
    many times (exact counting); codon_phased uses the reference's spaced
    seeds."""
    b = np.ascontiguousarray(bases, np.uint8)
    so = np.ascontiguousarray(seq_off, np.int64)
    ss = np.ascontiguousarray(sample_seqs, np.int64)
    km = np.ascontiguousarray(kmers, np.int32)
    n = len(ss) - 1
    words = np.zeros((n, len(km), s64 * bbits), np.uint64)
    inv = np.zeros((n, len(km)), np.float64)
    dens = np.zeros(n, np.uint8)
    lib.sko_sketch_samples(b.ctypes.data, so.ctypes.data, ss.ctypes.data, n, km.ctypes.data,
                           len(km), s64, bbits, int(use_rc), int(codon_phased), int(min_count),
                           words.ctypes.data, inv.ctypes.data, dens.ctypes.data, threads)
    return words, inv, dens.astype(bool)


def ref_available() -> bool:
    return REF_PATH.exists()


SKETCH_PATH = HERE / "_ref" / "libref_sketch.so"


class RefSketcher:
    """The reference's CPU sketcher (oracle/_ref/libref_sketch.so) and the
    seeded genome generator of the CPU parity case."""

    def __init__(self):
        if not SKETCH_PATH.exists():
            raise FileNotFoundError(f"{SKETCH_PATH} not built (needs the reference sources)")
        lib_ = C.CDLL(str(SKETCH_PATH))
        lib_.ref_make_genomes.restype = None
        lib_.ref_make_genomes.argtypes = [C.c_int, C.c_int64, C.c_uint64, C.c_void_p]
        lib_.ref_sketch_genomes.restype = C.c_int
        lib_.ref_sketch_genomes.argtypes = [C.c_void_p, C.c_int, C.c_int64, C.c_void_p, C.c_int,
                                            C.c_int, C.c_int, C.c_int, C.c_void_p]
        lib_.ref_sketch_file.restype = C.c_int
        lib_.ref_sketch_file.argtypes = [C.c_char_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                         C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        lib_.ref_seqbuf.restype = C.c_int
        lib_.ref_seqbuf.argtypes = [C.c_char_p, C.c_int, C.c_void_p, C.c_int64, C.c_void_p,
                                    C.c_int64, C.c_void_p, C.c_void_p]
        lib_.ref_sketch_seqs.restype = None
        lib_.ref_sketch_seqs.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                         C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                         C.c_void_p, C.c_void_p]
        self.lib = lib_

    def genomes(self, n, length, seed):
        out = np.empty((n, length), dtype=np.uint8)
        self.lib.ref_make_genomes(n, length, seed, out.ctypes.data)
        return out

    def sketch(self, genomes, kmers, s64, use_rc=True, threads=NTHREADS):
        g = np.ascontiguousarray(genomes, dtype=np.uint8)
        km = np.ascontiguousarray(kmers, np.int32)
        out = np.zeros((g.shape[0], len(km), s64 * 14), np.uint64)
        self.lib.ref_sketch_genomes(g.ctypes.data, g.shape[0], g.shape[1], km.ctypes.data, len(km),
                                    s64, int(use_rc), threads, out.ctypes.data)
        return out


    def sketch_seqs(self, bases, seq_off, sample_seqs, kmers, s64, use_rc=True, threads=NTHREADS,
                    codon_phased=False):
        """The reference's sketch() over samples of several sequences:
        words [n][K][s64*14], inv_minhash [n][K], densified [n]."""
        b = np.ascontiguousarray(bases, np.uint8)
        so = np.ascontiguousarray(seq_off, np.int64)
        ss = np.ascontiguousarray(sample_seqs, np.int64)
        km = np.ascontiguousarray(kmers, np.int32)
        n = len(ss) - 1
        words = np.zeros((n, len(km), s64 * 14), np.uint64)
        inv = np.zeros((n, len(km)), np.float64)
        dens = np.zeros(n, np.uint8)
        self.lib.ref_sketch_seqs(b.ctypes.data, so.ctypes.data, ss.ctypes.data, n, km.ctypes.data,
                                 len(km), s64, int(use_rc), int(codon_phased), threads,
                                 words.ctypes.data, inv.ctypes.data, dens.ctypes.data)
        return words, inv, dens.astype(bool)


    def sketch_file(self, path, kmers, s64, use_rc=True, min_count=0, exact=True):
        """The reference's SeqBuf + sketch() on one sequence file (one sample):
        (words [K][s64*14], inv_minhash [K], densified, is_reads)."""
        km = np.ascontiguousarray(kmers, np.int32)
        words = np.zeros((len(km), s64 * 14), np.uint64)
        inv = np.zeros(len(km), np.float64)
        dens = np.zeros(1, np.uint8)
        reads = self.lib.ref_sketch_file(str(path).encode(), km.ctypes.data, len(km), s64,
                                         int(use_rc), int(min_count), int(exact),
                                         words.ctypes.data, inv.ctypes.data, dens.ctypes.data)
        return words, inv, bool(dens[0]), bool(reads)


    def seqbuf(self, path, kmer_len, cap=1 << 26, cap_seqs=1 << 20):
        """What the reference's SeqBuf(files, kmer_len) keeps of one file:
        dict(seqs, total, missing_bases, reads, max_length, base_freq)."""
        bases = np.zeros(cap, np.uint8)
        off = np.zeros(cap_seqs + 1, np.int64)
        info = np.zeros(5, np.int64)
        freq = np.zeros(4, np.float64)
        rc = self.lib.ref_seqbuf(str(path).encode(), int(kmer_len), bases.ctypes.data, cap,
                                 off.ctypes.data, cap_seqs, info.ctypes.data, freq.ctypes.data)
        if rc != 0:
            raise ValueError("ref_seqbuf capacity too small")
        n = int(info[0])
        seqs = [bytes(bases[off[i]:off[i + 1]]).decode() for i in range(n)]
        return {"seqs": seqs, "total": int(info[1]), "missing_bases": int(info[2]),
                "reads": bool(info[3]), "max_length": int(info[4]), "base_freq": freq.tolist()}


def sketcher_available() -> bool:
    return SKETCH_PATH.exists()


REF_GPU_PATH = HERE / "_ref" / "libref_gpu.so"


class RefGpuKernel:
    """The reference's own GPU distance kernel (`calculate_dists`,
    src/gpu/dist.cu:164-317), compiled for sm_100a from the reference sources
    and launched by oracle/ref_gpu_dists.cu the way dispatchDists does
    (src/gpu/dist.cu:408-470).  Baseline on the same GPU; not the checker of
    record (its float regression and first-low-k truncation differ from the
    reference's CPU semantics)."""

    def __init__(self):
        if not REF_GPU_PATH.exists():
            raise FileNotFoundError(f"{REF_GPU_PATH} not built (needs the reference sources)")
        lib_ = C.CDLL(str(REF_GPU_PATH))
        lib_.refgpu_dists.restype = C.c_int
        lib_.refgpu_dists.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p,
                                      C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                      C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                      C.POINTER(C.c_double), C.c_char_p, C.c_int]
        lib_.refgpu_self_dists.restype = C.c_int
        lib_.refgpu_self_dists.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int, C.c_int,
                                           C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                           C.POINTER(C.c_double), C.c_char_p, C.c_int]
        self.lib = lib_

    def self_dists(self, words, kmers, s64, random_k=None, warmup=0, launches=1, want_out=True,
                   bbits=14):
        """All-vs-all (core, accessory) of `words` [n][K][s64*bbits]: returns
        (float32 (n(n-1)/2, 2) or None, mean ms per timed launch)."""
        w = np.ascontiguousarray(words, np.uint64)
        n = w.shape[0]
        km = np.ascontiguousarray(kmers, np.int32)
        rk = None if random_k is None else np.ascontiguousarray(random_k, np.float32)
        out = np.zeros((n * (n - 1) // 2, 2), np.float32) if want_out else None
        ms = C.c_double(0.0)
        err = C.create_string_buffer(512)
        rc = self.lib.refgpu_self_dists(w.ctypes.data, n, km.ctypes.data, len(km), s64, bbits,
                                        None if rk is None else rk.ctypes.data, warmup, launches,
                                        None if out is None else out.ctypes.data, C.byref(ms),
                                        err, len(err))
        if rc != 0:
            raise RuntimeError(err.value.decode())
        return out, ms.value


    def dists(self, ref_words, kmers, s64, query_words=None, table=None, ref_lookup=None,
              query_lookup=None, bbits=14):
        """(core, accessory) float32 (n_pairs, 2) of the reference kernel.
        table: None (NoAdjust), float [K] (one chance per k) or [K][C][C]
        with uint16 cluster lookups (RandomMC::flattened_random strides)."""
        r = np.ascontiguousarray(ref_words, np.uint64)
        q = None if query_words is None else np.ascontiguousarray(query_words, np.uint64)
        km = np.ascontiguousarray(kmers, np.int32)
        n_ref = r.shape[0]
        n_q = 0 if q is None else q.shape[0]
        pairs = n_ref * (n_ref - 1) // 2 if q is None else n_ref * n_q
        t = None if table is None else np.ascontiguousarray(table, np.float32)
        n_cl = 0 if t is None or t.ndim == 1 else t.shape[1]
        rl = None if ref_lookup is None else np.ascontiguousarray(ref_lookup, np.uint16)
        ql = None if query_lookup is None else np.ascontiguousarray(query_lookup, np.uint16)
        out = np.zeros((pairs, 2), np.float32)
        ms = C.c_double(0.0)
        err = C.create_string_buffer(512)
        ptr = lambda a: None if a is None else a.ctypes.data
        rc = self.lib.refgpu_dists(r.ctypes.data, n_ref, ptr(q), n_q, km.ctypes.data, len(km), s64,
                                   bbits, ptr(t), n_cl, ptr(rl), ptr(ql), 0, 1, out.ctypes.data,
                                   C.byref(ms), err, len(err))
        if rc != 0:
            raise RuntimeError(err.value.decode())
        return out


def ref_gpu_available() -> bool:
    return REF_GPU_PATH.exists()
