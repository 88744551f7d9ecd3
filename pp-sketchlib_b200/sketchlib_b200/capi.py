"""ctypes binding of the C ABI in include/sketchlib_b200.h.

This is the thinnest possible host layer over the library: each wrapper
checks the returned sk_status and raises with the library's message.  Arrays
are numpy on the host; device buffers are passed as integer addresses (for
example ``torch.Tensor.data_ptr()``).

The shared library is required: importing this module raises if
``libsketchlib_b200.so`` is missing, there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().with_name("libsketchlib_b200.so")

SK_OK, SK_EINVAL, SK_ENOMEM, SK_ECUDA, SK_EMISMATCH = 0, 1, 2, 3, 4
SK_ECANCELLED, SK_ETIMEDOUT, SK_ENOTSUP, SK_EKERNEL, SK_ERANGE = 5, 6, 7, 8, 9
STATUS_NAMES = {
    0: "SK_OK", 1: "SK_EINVAL", 2: "SK_ENOMEM", 3: "SK_ECUDA", 4: "SK_EMISMATCH",
    5: "SK_ECANCELLED", 6: "SK_ETIMEDOUT", 7: "SK_ENOTSUP", 8: "SK_EKERNEL", 9: "SK_ERANGE",
}
RANDOM_NONE, RANDOM_EQUAL_BASE, RANDOM_TABLE = 0, 1, 2
SEMANTICS_REFERENCE_CPU, SEMANTICS_REFERENCE_GPU = 0, 1
OUT_CORE_ACC, OUT_JACCARD, OUT_COUNTS = 0, 1, 2

_p = C.c_void_p
_i32, _i64, _u64, _f32 = C.c_int32, C.c_int64, C.c_uint64, C.c_float

# name: (restype, argtypes)
_SIGNATURES = {
    "sk_abi_version": (_i32, []),
    "sk_ctx_create": (_i32, [_i32, C.POINTER(_p)]),
    "sk_ctx_destroy": (_i32, [_p]),
    "sk_last_error": (C.c_char_p, [_p]),
    "sk_ctx_set_stream": (_i32, [_p, _p]),
    "sk_cancel": (_i32, [_p]),
    "sk_device_info": (_i32, [_p, C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_i32)]),
    "sk_ctx_synchronize": (_i32, [_p]),
    "sk_ctx_set_tile_config": (_i32, [_p, _i32]),
    "sk_ctx_set_semantics": (_i32, [_p, _i32]),
    "sk_ctx_set_memory_limit": (_i32, [_p, _i64]),
    "sk_tile_config_count": (_i32, []),
    "sk_tile_config_info": (_i32, [_i32] + [C.POINTER(_i32)] * 5),
    "sk_ctx_load_tuning": (_i32, [_p, C.c_char_p]),
    "sk_db_create": (_i32, [_p, _p, _i64, _p, _i32, _i32, _i32, C.POINTER(_p)]),
    "sk_db_create_device": (_i32, [_p, _p, _i64, _p, _i32, _i32, _i32, C.POINTER(_p)]),
    "sk_db_destroy": (_i32, [_p]),
    "sk_db_info": (_i32, [_p, C.POINTER(_i64), C.POINTER(_i32), C.POINTER(_i32), C.POINTER(_i32)]),
    "sk_db_set_sample_info": (_i32, [_p, _p, _p]),
    "sk_db_download": (_i32, [_p, _p, _p]),
    "sk_random_create": (_i32, [_p, _i32, _i32, _p, _i32, _i32, _p, C.POINTER(_p)]),
    "sk_random_destroy": (_i32, [_p]),
    "sk_closest_cluster": (_i32, [_p, _i32, _i32, _p, _i64, _p]),
    "sk_random_set_centroids": (_i32, [_p, _p, _i32]),
    "sk_dists_rows": (_i64, [_p, _p]),
    "sk_dists_dense": (_i32, [_p, _p, _p, _p, _i32, _p, _i32]),
    "sk_query_db": (_i32, [_p, _p, _p, _p, _i32, _i32, _i32, _p, _i32, _p]),
    "sk_query_db_ready": (_i32, [_p, _p, _p, _p, _i32, _i32, _i32, _p, _i32, _p, _p, _p]),
    "sk_dists_knn": (_i32, [_p, _p, _p, _i32, _i32, _i32, _p, _p, _p]),
    "sk_query_knn": (_i32, [_p, _p, _p, _p, _i32, _i32, _p, _p]),
    "sk_sparse_threshold": (_i32, [_p, _p, _i64, _i32, _i32, _f32, C.POINTER(_p)]),
    "sk_dists_threshold": (_i32, [_p, _p, _p, _i32, _f32, C.POINTER(_p)]),
    "sk_sparse_size": (_i64, [_p]),
    "sk_sparse_copy": (_i32, [_p, _p, _p, _p]),
    "sk_sparse_destroy": (_i32, [_p]),
    "sk_long_to_square": (_i32, [_p, _p, _i64, _p, _p, _i64, _p]),
    "sk_square_to_long": (_i32, [_p, _p, _i64, _p]),
    "sk_synth_host": (_i32, [_p, _p, _i64, _i32, _i32, _u64, _i32, _p]),
    "sk_synth_device": (_i32, [_p, _p, _p, _i64, _i32, _i32, _u64, _p]),
    "sk_probe_alu_peak": (_i32, [_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "sk_probe_wait_limit": (_i32, [_p, _i32]),
    "sk_batch_create": (_i32, [_p, _p, _i32, _i32, C.POINTER(_p)]),
    "sk_batch_run": (_i32, [_p]),
    "sk_batch_launch": (_i32, [_p]),
    "sk_batch_info": (_i32, [_p, C.POINTER(_i32), C.POINTER(_i32), C.POINTER(_i64),
                             C.POINTER(_i64)]),
    "sk_batch_destroy": (_i32, [_p]),
    "sk_autotune": (_i32, [_p, _p, _p, _p, _i32, C.POINTER(_i32)]),
    "sk_ctx_save_tuning": (_i32, [_p, C.c_char_p]),
    "sk_dists_dense_noalloc": (_i32, [_p, _p, _p, _p, _i32, _p]),
    "sk_host_alloc": (_i32, [_i64, C.POINTER(_p)]),
    "sk_host_free": (_i32, [_p]),
    "sk_server_create": (_i32, [_p, _p, _p, _p, C.POINTER(_p)]),
    "sk_server_submit": (_i32, [_p, _p, _i64, _p, _p, _p, C.POINTER(_i64)]),
    "sk_server_wait": (_i32, [_p, _i64, C.c_double]),
    "sk_server_result": (_i32, [_p, _i64, _p, _p, _p, C.POINTER(C.c_double)]),
    "sk_server_release": (_i32, [_p, _i64]),
    "sk_server_stats": (_i32, [_p, C.POINTER(_i64), C.POINTER(C.c_double), C.POINTER(_i64)]),
    "sk_server_info": (_i32, [_p, C.POINTER(_i32), C.POINTER(_i64), C.POINTER(_i64),
                               C.POINTER(_i64)]),
    "sk_server_destroy": (_i32, [_p]),
    "sk_sketch": (_i32, [_p, _p, _p, _p, _i64, _p, _i32, _i32, _i32, _i32, _i32, _p, _p, _p]),
    "sk_sketch_device": (_i32, [_p, _p, _p, _p, _i64, _p, _i32, _i32, _i32, _i32, _i32, _p, _p,
                                _p]),
}


class ServerParams(C.Structure):
    _fields_ = [("slots", _i32), ("slice_queries", _i32), ("kNN", _i32), ("dist_col", _i32),
                ("keep_rows", _i32), ("large_slice_queries", _i32), ("device_bytes", _i64)]

BATCH_AUTOTUNE = 1


class HostSketches(C.Structure):
    """sk_host_sketches: one side of an sk_query_db call."""
    _fields_ = [("words", _p), ("n", _i64), ("cluster", _p), ("seq_len", _p)]


class Job(C.Structure):
    """sk_job: one distance job of a batch (outputs in device memory)."""
    _fields_ = [("ref", _p), ("query", _p), ("random", _p), ("out_mode", _i32), ("out", _p)]

# Entry points a newer header may add; bound when the library exports them.
_OPTIONAL = {}


class SketchlibError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def _load() -> C.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python pp-sketchlib_b200/build.py` "
            "(there is no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    for name, (res, args) in _OPTIONAL.items():
        if hasattr(lib, name):
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
    return lib


lib = _load()


def _ptr(a) -> int | None:
    if a is None:
        return None
    if isinstance(a, int):
        return a
    return a.ctypes.data


def _check(status: int, ctx=None):
    if status != SK_OK:
        msg = lib.sk_last_error(ctx.handle).decode() if ctx is not None and ctx.handle else ""
        raise SketchlibError(status, msg)


def exported_symbols() -> list[str]:
    return list(_SIGNATURES)


class Context:
    """A device plus its stream (sk_ctx)."""

    def __init__(self, device_id: int = 0):
        h = _p()
        st = lib.sk_ctx_create(device_id, C.byref(h))
        if st != SK_OK:
            raise SketchlibError(st, f"cannot create a context on device {device_id}")
        self.handle = h.value

    def close(self):
        if self.handle:
            lib.sk_ctx_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def last_error(self) -> str:
        return lib.sk_last_error(self.handle).decode()

    def device_info(self):
        f, t, s = _i64(), _i64(), _i32()
        _check(lib.sk_device_info(self.handle, C.byref(f), C.byref(t), C.byref(s)), self)
        return f.value, t.value, s.value

    def synchronize(self):
        _check(lib.sk_ctx_synchronize(self.handle), self)

    def set_stream(self, stream_handle: int):
        _check(lib.sk_ctx_set_stream(self.handle, stream_handle), self)

    def set_tile_config(self, config_id: int):
        _check(lib.sk_ctx_set_tile_config(self.handle, config_id), self)

    def set_semantics(self, semantics: int):
        """SEMANTICS_REFERENCE_CPU (default) or SEMANTICS_REFERENCE_GPU: which
        reference path the core/accessory fit reproduces (sk_ctx_set_semantics)."""
        _check(lib.sk_ctx_set_semantics(self.handle, semantics), self)

    def set_memory_limit(self, nbytes: int):
        """Device bytes a dense call to host memory may stage its output in
        (0 = free memory less 2 GiB); larger outputs are computed in row blocks."""
        _check(lib.sk_ctx_set_memory_limit(self.handle, nbytes), self)

    def load_tuning(self, path: str):
        _check(lib.sk_ctx_load_tuning(self.handle, str(path).encode()), self)

    def cancel(self):
        lib.sk_cancel(self.handle)


def closest_cluster(centroids, base_freq, use_rc: bool = True) -> np.ndarray:
    """Random-match cluster of each sample from its A, C, G, T frequencies
    (sk_closest_cluster): the nearest centroid [C][4] after averaging A/T and
    C/G when the strand is unknown (use_rc)."""
    c = np.ascontiguousarray(centroids, np.float32).reshape(-1, 4)
    b = np.ascontiguousarray(base_freq, np.float64).reshape(-1, 4)
    out = np.zeros(b.shape[0], np.uint16)
    st = lib.sk_closest_cluster(c.ctypes.data, c.shape[0], int(use_rc), b.ctypes.data,
                                b.shape[0], out.ctypes.data)
    if st != SK_OK:
        raise SketchlibError(st, "closest_cluster: bad arguments")
    return out


def probe_alu_peak(ctx: Context) -> tuple[float, float]:
    """Measured (LOP3/s, POPC/s) of the context's device."""
    l, p = C.c_double(), C.c_double()
    _check(lib.sk_probe_alu_peak(ctx.handle, C.byref(l), C.byref(p)), ctx)
    return l.value, p.value


def tile_configs() -> list[dict]:
    out = []
    for cid in range(1, lib.sk_tile_config_count() + 1):
        v = [_i32() for _ in range(5)]
        if lib.sk_tile_config_info(cid, *[C.byref(x) for x in v]) == SK_OK:
            out.append(dict(id=cid, tile_rows=v[0].value, tile_cols=v[1].value,
                            thread_rows=v[2].value, thread_cols=v[3].value,
                            max_kmers=v[4].value))
    return out


class Database:
    """Sketches resident on the device (sk_db).

    words: uint64 array [n_samples, n_kmers, sketchsize64 * 14] in the
    reference's word layout, or an integer device address with n_samples given.
    """

    def __init__(self, ctx: Context, words, kmers, sketchsize64: int, bbits: int = 14,
                 n_samples: int | None = None, cluster=None, seq_len=None):
        self.ctx = ctx
        kmers_arr = np.ascontiguousarray(kmers, dtype=np.int32)
        h = _p()
        if isinstance(words, int):
            if n_samples is None:
                raise ValueError("n_samples is required with a device address")
            st = lib.sk_db_create_device(ctx.handle, words, n_samples, kmers_arr.ctypes.data,
                                         len(kmers_arr), sketchsize64, bbits, C.byref(h))
            n = n_samples
        else:
            w = np.ascontiguousarray(words, dtype=np.uint64)
            n = w.shape[0]
            if w.size != n * len(kmers_arr) * sketchsize64 * bbits:
                raise ValueError("words do not match n_kmers * sketchsize64 * bbits per sample")
            st = lib.sk_db_create(ctx.handle, w.ctypes.data, n, kmers_arr.ctypes.data,
                                  len(kmers_arr), sketchsize64, bbits, C.byref(h))
        _check(st, ctx)
        self.handle = h.value
        self.n = n
        self.kmers = kmers_arr
        self.sketchsize64 = sketchsize64
        self.bbits = bbits
        if cluster is not None or seq_len is not None:
            self.set_sample_info(cluster, seq_len)

    def set_sample_info(self, cluster=None, seq_len=None):
        cl = None if cluster is None else np.ascontiguousarray(cluster, dtype=np.uint16)
        ln = None if seq_len is None else np.ascontiguousarray(seq_len, dtype=np.uint64)
        _check(lib.sk_db_set_sample_info(self.handle, _ptr(cl), _ptr(ln)), self.ctx)

    def download(self) -> np.ndarray:
        out = np.empty((self.n, len(self.kmers), self.sketchsize64 * self.bbits), dtype=np.uint64)
        _check(lib.sk_db_download(self.ctx.handle, self.handle, out.ctypes.data), self.ctx)
        return out

    def close(self):
        if self.handle:
            lib.sk_db_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Random:
    """Random-match correction model (sk_random)."""

    def __init__(self, ctx: Context, mode: int, kmers, use_rc: bool = True, table=None):
        self.ctx = ctx
        kmers_arr = np.ascontiguousarray(kmers, dtype=np.int32)
        tab = None
        n_clusters = 0
        if table is not None:
            tab = np.ascontiguousarray(table, dtype=np.float32)
            n_clusters = tab.shape[-1]
        h = _p()
        _check(lib.sk_random_create(ctx.handle, mode, int(use_rc), kmers_arr.ctypes.data,
                                    len(kmers_arr), n_clusters, _ptr(tab), C.byref(h)), ctx)
        self.handle = h.value
        self.mode = mode

    def set_centroids(self, centroids):
        """Base-composition centroids [C][4] (A, C, G, T) of a table model, for
        the server's cluster assignment of queries."""
        c = np.ascontiguousarray(centroids, dtype=np.float32)
        _check(lib.sk_random_set_centroids(self.handle, c.ctypes.data, c.shape[0]), self.ctx)

    def close(self):
        if self.handle:
            lib.sk_random_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _h(x):
    return None if x is None else x.handle


class Batch:
    """A captured persistent launch over many jobs (sk_batch).

    jobs: list of (ref Database, query Database or None, Random or None,
    out_mode, device address of the output)."""

    def __init__(self, ctx: Context, jobs, autotune: bool = False):
        self.ctx = ctx
        self._keep = list(jobs)
        arr = (Job * len(jobs))()
        for i, (ref, query, rnd, mode, out) in enumerate(jobs):
            arr[i] = Job(ref.handle, _h(query), _h(rnd), mode, out)
        h = _p()
        _check(lib.sk_batch_create(ctx.handle, C.cast(arr, _p), len(jobs),
                                   BATCH_AUTOTUNE if autotune else 0, C.byref(h)), ctx)
        self.handle = h.value

    def run(self):
        _check(lib.sk_batch_run(self.handle), self.ctx)

    def launch(self):
        _check(lib.sk_batch_launch(self.handle), self.ctx)

    def info(self) -> dict:
        c, g, n, p = _i32(), _i32(), _i64(), _i64()
        _check(lib.sk_batch_info(self.handle, C.byref(c), C.byref(g), C.byref(n), C.byref(p)),
               self.ctx)
        return dict(tile_config=c.value, grid=g.value, n_items=n.value, n_pairs=p.value)

    def close(self):
        if self.handle:
            lib.sk_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """A query server over a resident reference database (sk_server)."""

    def __init__(self, ctx: Context, ref: Database, random: Random | None = None, slots: int = 3,
                 slice_queries: int = 128, kNN: int = 5, dist_col: int = 0,
                 keep_rows: bool = False, large_slice_queries: int = 0,
                 device_bytes: int = 0):
        self.ctx = ctx
        self.ref = ref
        self.kNN = kNN
        self.keep_rows = keep_rows
        self._inputs = {}
        prm = ServerParams(slots, slice_queries, kNN, dist_col, int(keep_rows),
                           large_slice_queries, device_bytes)
        h = _p()
        _check(lib.sk_server_create(ctx.handle, ref.handle, _h(random), C.byref(prm), C.byref(h)),
               ctx)
        self.handle = h.value

    def submit(self, words, cluster=None, seq_len=None, base_freq=None) -> int:
        w = np.ascontiguousarray(words, dtype=np.uint64)
        cl = None if cluster is None else np.ascontiguousarray(cluster, np.uint16)
        ln = None if seq_len is None else np.ascontiguousarray(seq_len, np.uint64)
        bf = None if base_freq is None else np.ascontiguousarray(base_freq, np.float64)
        if bf is not None and bf.shape != (w.shape[0], 4):
            raise ValueError("base_freq must be [n_queries][4]")
        t = _i64()
        st = lib.sk_server_submit(self.handle, w.ctypes.data, w.shape[0], _ptr(cl), _ptr(ln),
                                  _ptr(bf), C.byref(t))
        if st != SK_OK:
            raise SketchlibError(st, "submit failed")
        self._inputs[t.value] = (w, cl, ln)       # the server reads them until done
        return t.value

    def wait(self, ticket: int, timeout: float = 60.0):
        st = lib.sk_server_wait(self.handle, ticket, timeout)
        if st != SK_OK:
            raise SketchlibError(st, f"request {ticket} did not complete")

    def result(self, ticket: int, release: bool = True):
        n = self._inputs[ticket][0].shape[0]
        idx = np.empty((n, self.kNN), np.int64)
        dist = np.empty((n, self.kNN), np.float32)
        rows = np.empty((n, self.ref.n, 2), np.float32) if self.keep_rows else None
        lat = C.c_double()
        st = lib.sk_server_result(self.handle, ticket, idx.ctypes.data, dist.ctypes.data,
                                  _ptr(rows), C.byref(lat))
        if st != SK_OK:
            raise SketchlibError(st, f"request {ticket} failed")
        if release:
            lib.sk_server_release(self.handle, ticket)
            self._inputs.pop(ticket, None)
        return idx, dist, rows, lat.value

    def stats(self):
        p, u, q = _i64(), C.c_double(), _i64()
        _check(lib.sk_server_stats(self.handle, C.byref(p), C.byref(u), C.byref(q)), self.ctx)
        return dict(pairs_done=p.value, uptime_s=u.value, queued_queries=q.value)

    def info(self):
        n, b, sl, sh = _i32(), _i64(), _i64(), _i64()
        _check(lib.sk_server_info(self.handle, C.byref(n), C.byref(b), C.byref(sl), C.byref(sh)),
               self.ctx)
        return dict(slots=n.value, slot_bytes=b.value, slices=sl.value, slices_shared=sh.value)

    def close(self):
        if self.handle:
            lib.sk_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(ctx: Context, ref: Database, query: Database | None = None,
             random: Random | None = None, repeats: int = 2) -> int:
    best = _i32()
    _check(lib.sk_autotune(ctx.handle, ref.handle, _h(query), _h(random), repeats,
                           C.byref(best)), ctx)
    return best.value


def save_tuning(ctx: Context, path: str):
    _check(lib.sk_ctx_save_tuning(ctx.handle, str(path).encode()), ctx)


def dists_rows(ref: Database, query: Database | None = None) -> int:
    return lib.sk_dists_rows(ref.handle, _h(query))


def dists_dense(ctx: Context, ref: Database, query: Database | None = None,
                random: Random | None = None, out_mode: int = OUT_CORE_ACC,
                out=None) -> np.ndarray | None:
    """Dense long-form distances.  With `out` an integer device address the
    call only queues the kernels (returns None); otherwise returns numpy."""
    rows = dists_rows(ref, query)
    K = len(ref.kmers)
    if isinstance(out, int):
        _check(lib.sk_dists_dense(ctx.handle, ref.handle, _h(query), _h(random), out_mode, out, 1), ctx)
        return None
    if out is None:
        if out_mode == OUT_CORE_ACC:
            out = np.empty((rows, 2), dtype=np.float32)
        elif out_mode == OUT_JACCARD:
            out = np.empty((rows, K), dtype=np.float32)
        else:
            out = np.empty((rows, K), dtype=np.uint32)
    _check(lib.sk_dists_dense(ctx.handle, ref.handle, _h(query), _h(random), out_mode,
                              out.ctypes.data, 0), ctx)
    return out


def query_db(ctx: Context, ref_words, kmers, sketchsize64: int, query_words=None,
             ref_cluster=None, ref_seq_len=None, query_cluster=None, query_seq_len=None,
             random: Random | None = None, out_mode: int = OUT_CORE_ACC, out=None,
             bbits: int = 14, ready=None) -> np.ndarray:
    """Host sketches in, host distances out (sk_query_db): the upload is
    chunked and overlapped with the distance kernel.  `ref_words` /
    `query_words`: uint64 [n][K][sketchsize64 * bbits]; query_words None =
    all-vs-all.  Pinned arrays (e.g. from torch's pin_memory) copy fastest.
    ready(side, s0, n) -> bool, if given, is asked before each chunk of
    samples is copied (side 0 ref, 1 query) and returns once its words are in
    place (sk_query_db_ready); False abandons the call."""
    keep = []

    def side(words, cluster, seq_len):
        w = words if isinstance(words, np.ndarray) and words.dtype == np.uint64 and \
            words.flags.c_contiguous else np.ascontiguousarray(words, dtype=np.uint64)
        cl = None if cluster is None else np.ascontiguousarray(cluster, np.uint16)
        ln = None if seq_len is None else np.ascontiguousarray(seq_len, np.uint64)
        keep.extend([w, cl, ln])
        return HostSketches(w.ctypes.data, w.shape[0], _ptr(cl), _ptr(ln)), w.shape[0]

    r, n_ref = side(ref_words, ref_cluster, ref_seq_len)
    q, n_q = (None, 0) if query_words is None else side(query_words, query_cluster, query_seq_len)
    K = len(kmers)
    rows = n_ref * (n_ref - 1) // 2 if q is None else n_q * n_ref
    if out is None:
        if out_mode == OUT_CORE_ACC:
            out = np.empty((rows, 2), dtype=np.float32)
        elif out_mode == OUT_JACCARD:
            out = np.empty((rows, K), dtype=np.float32)
        else:
            out = np.empty((rows, K), dtype=np.uint32)
    km = np.ascontiguousarray(kmers, np.int32)
    if ready is None:
        _check(lib.sk_query_db(ctx.handle, C.byref(r), None if q is None else C.byref(q),
                               km.ctypes.data, K, sketchsize64, bbits, _h(random), out_mode,
                               out.ctypes.data), ctx)
        return out
    cb = _READY_FN(lambda user, side, s0, n: 0 if ready(side, s0, n) else 1)
    _check(lib.sk_query_db_ready(ctx.handle, C.byref(r), None if q is None else C.byref(q),
                                 km.ctypes.data, K, sketchsize64, bbits, _h(random), out_mode,
                                 out.ctypes.data, C.cast(cb, C.c_void_p), None), ctx)
    return out


# sk_words_ready_fn
_READY_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int32, C.c_int64, C.c_int64)


def pack_sequences(samples):
    """Samples as lists of sequences (str or bytes) -> (bases uint8,
    seq_offsets int64 [n_seqs + 1], sample_seqs int64 [n_samples + 1]), the
    flat form sk_sketch takes."""
    seqs = [q.encode() if isinstance(q, str) else bytes(q) for smp in samples for q in smp]
    seq_off = np.zeros(len(seqs) + 1, np.int64)
    np.cumsum([len(q) for q in seqs], out=seq_off[1:])
    sample_seqs = np.zeros(len(samples) + 1, np.int64)
    np.cumsum([len(smp) for smp in samples], out=sample_seqs[1:])
    bases = np.frombuffer(b"".join(seqs), np.uint8) if seqs else np.zeros(0, np.uint8)
    return bases, seq_off, sample_seqs


def sketch(ctx: Context, bases, seq_offsets, sample_seqs, kmers, sketchsize64: int,
           use_rc: bool = True, min_count: int = 0, words=None, codon_phased: bool = False):
    """MinHash sketches of sequences on the device (sk_sketch).  `bases`
    uint8 (or bytes) holding every sequence back to back; sequence i is
    bases[seq_offsets[i]:seq_offsets[i+1]]; sample s owns sequences
    sample_seqs[s] .. sample_seqs[s+1]-1; codon_phased selects the reference's
    spaced seeds.  Returns (words uint64 [n][K][sketchsize64 * 14],
    inv_minhash float64 [n][K], densified bool [n])."""
    b = np.frombuffer(bases, np.uint8) if isinstance(bases, (bytes, bytearray)) else \
        np.ascontiguousarray(bases, np.uint8)
    so = np.ascontiguousarray(seq_offsets, np.int64)
    ss = np.ascontiguousarray(sample_seqs, np.int64)
    km = np.ascontiguousarray(kmers, np.int32)
    n = len(ss) - 1
    if words is None:
        words = np.empty((n, len(km), sketchsize64 * 14), np.uint64)
    inv = np.empty((n, len(km)), np.float64)
    dens = np.empty(n, np.uint8)
    _check(lib.sk_sketch(ctx.handle, b.ctypes.data if b.size else None, so.ctypes.data,
                         ss.ctypes.data, n, km.ctypes.data, len(km), sketchsize64, int(use_rc),
                         int(codon_phased), int(min_count), words.ctypes.data, inv.ctypes.data,
                         dens.ctypes.data), ctx)
    return words, inv, dens.astype(bool)


def sketch_device(ctx: Context, d_bases: int, seq_offsets, sample_seqs, kmers, sketchsize64: int,
                  d_words: int, use_rc: bool = True, min_count: int = 0, d_inv_minhash: int = 0,
                  d_densified: int = 0, codon_phased: bool = False) -> None:
    """sk_sketch_device: device bases in (address d_bases), device outputs
    (addresses d_words [n][K][sketchsize64 * 14] uint64, d_inv_minhash [n][K]
    float64 and d_densified [n] uint8, 0 to skip); e.g. torch tensors'
    data_ptr().  Offsets are host arrays as for sketch()."""
    so = np.ascontiguousarray(seq_offsets, np.int64)
    ss = np.ascontiguousarray(sample_seqs, np.int64)
    km = np.ascontiguousarray(kmers, np.int32)
    _check(lib.sk_sketch_device(ctx.handle, d_bases or None, so.ctypes.data, ss.ctypes.data,
                                len(ss) - 1, km.ctypes.data, len(km), sketchsize64, int(use_rc),
                                int(codon_phased), int(min_count), d_words, d_inv_minhash or None,
                                d_densified or None), ctx)


def dists_knn(ctx: Context, db: Database, kNN: int, dist_col: int = 0, jaccard: bool = False,
              random: Random | None = None):
    n = db.n
    i = np.empty(n * kNN, dtype=np.int64)
    j = np.empty(n * kNN, dtype=np.int64)
    d = np.empty(n * kNN, dtype=np.float32)
    _check(lib.sk_dists_knn(ctx.handle, db.handle, _h(random), kNN, dist_col, int(jaccard),
                            i.ctypes.data, j.ctypes.data, d.ctypes.data), ctx)
    return i, j, d


def query_knn(ctx: Context, ref: Database, query: Database, kNN: int, dist_col: int = 0,
              random: Random | None = None):
    r = np.empty((query.n, kNN), dtype=np.int64)
    d = np.empty((query.n, kNN), dtype=np.float32)
    _check(lib.sk_query_knn(ctx.handle, ref.handle, query.handle, _h(random), kNN, dist_col,
                            r.ctypes.data, d.ctypes.data), ctx)
    return r, d


def _sparse_take(ctx, h):
    try:
        n = lib.sk_sparse_size(h)
        i = np.empty(n, dtype=np.int64)
        j = np.empty(n, dtype=np.int64)
        d = np.empty(n, dtype=np.float32)
        _check(lib.sk_sparse_copy(h, i.ctypes.data, j.ctypes.data, d.ctypes.data), ctx)
        return i, j, d
    finally:
        lib.sk_sparse_destroy(h)


def sparse_threshold(ctx: Context, long_form: np.ndarray, n_samples: int, col: int,
                     cutoff: float):
    lf = np.ascontiguousarray(long_form, dtype=np.float32)
    if lf.ndim == 1:
        lf = lf.reshape(-1, 1)
    h = _p()
    _check(lib.sk_sparse_threshold(ctx.handle, lf.ctypes.data, n_samples, lf.shape[1], col,
                                   float(cutoff), C.byref(h)), ctx)
    return _sparse_take(ctx, h.value)


def dists_threshold(ctx: Context, db: Database, dist_col: int, cutoff: float,
                    random: Random | None = None):
    h = _p()
    _check(lib.sk_dists_threshold(ctx.handle, db.handle, _h(random), dist_col, float(cutoff),
                                  C.byref(h)), ctx)
    return _sparse_take(ctx, h.value)


def long_to_square(ctx: Context, rr, qr=None, qq=None, n_qq: int = 0) -> np.ndarray:
    rr = np.ascontiguousarray(rr, dtype=np.float32).ravel()
    n_rr = int(round(0.5 * (1 + np.sqrt(1 + 8 * rr.size)))) if rr.size else (1 if n_qq else 0)
    qr_a = None if qr is None else np.ascontiguousarray(qr, dtype=np.float32).ravel()
    qq_a = None if qq is None else np.ascontiguousarray(qq, dtype=np.float32).ravel()
    n = n_rr + n_qq
    out = np.empty((n, n), dtype=np.float32)
    _check(lib.sk_long_to_square(ctx.handle, rr.ctypes.data, n_rr, _ptr(qr_a), _ptr(qq_a), n_qq,
                                 out.ctypes.data), ctx)
    return out


def square_to_long(ctx: Context, square) -> np.ndarray:
    sq = np.ascontiguousarray(square, dtype=np.float32)
    if sq.ndim != 2 or sq.shape[0] != sq.shape[1]:
        raise SketchlibError(1, "square_to_long input must be a square matrix")
    n = sq.shape[0]
    out = np.empty(n * (n - 1) // 2, dtype=np.float32)
    _check(lib.sk_square_to_long(ctx.handle, sq.ctypes.data, n, out.ctypes.data), ctx)
    return out


def synth_host(parent, thresh, sketchsize64: int, seed: int, threads: int = 8) -> np.ndarray:
    par = np.ascontiguousarray(parent, dtype=np.int32)
    th = np.ascontiguousarray(thresh, dtype=np.uint32)
    n, K = th.shape
    out = np.empty((n, K, sketchsize64 * 14), dtype=np.uint64)
    st = lib.sk_synth_host(par.ctypes.data, th.ctypes.data, n, K, sketchsize64, seed, threads,
                           out.ctypes.data)
    if st != SK_OK:
        raise SketchlibError(st, "sk_synth_host failed")
    return out


def synth_device(ctx: Context, parent, thresh, sketchsize64: int, seed: int, d_words: int):
    par = np.ascontiguousarray(parent, dtype=np.int32)
    th = np.ascontiguousarray(thresh, dtype=np.uint32)
    n, K = th.shape
    _check(lib.sk_synth_device(ctx.handle, par.ctypes.data, th.ctypes.data, n, K, sketchsize64,
                               seed, d_words), ctx)
