"""Minimal writer of pp-sketchlib sketch databases (test fixtures).

Writes the classic HDF5 layout the reference produces through HighFive
(superblock v0, version-1 object headers, symbol-table groups, contiguous
datasets, attributes in header messages, variable-length strings in a global
heap), following the published HDF5 file-format specification, so tests can
build `<name>.h5` databases on machines without h5py and drive the drop-in
`pp_sketchlib.queryDatabase` end to end.

Layout written (src/database/database.cpp:48-112, 150-190):
  /sketches                 attrs sketch_version (string), codon_phased (u8), reverse_complement (u8)
  /sketches/<sample>        attrs sketchsize64, bbits, length, missing_bases (u64), reads (u8),
                            base_freq (f64[4]), kmers (i32[K])
  /sketches/<sample>/<k>    u64[sketchsize64 * bbits], attr kmer-size (i32)
  /random (optional)        attrs k_min, k_max (u32), use_rc (u8); datasets table_keys (vlen str),
                            table_values (u16), matches_keys (u64), matches_values (f32, attr dims
                            u64[3]), centroids (f32, attr dims u64[2])
"""
from __future__ import annotations

import struct

import numpy as np

UNDEF = 0xFFFFFFFFFFFFFFFF
LEAF_K = 64        # up to 128 links per symbol-table node
INTERNAL_K = 64    # up to 128 symbol-table nodes under the group's B-tree node


def _pad8(b: bytes) -> bytes:
    return b + b"\0" * (-len(b) % 8)


# ------------------------------------------------------------ datatypes

def _dt_int(size: int, signed: bool) -> bytes:
    return bytes([0x10, 0x08 if signed else 0, 0, 0]) + struct.pack("<IHH", size, 0, size * 8)


def _dt_float(size: int) -> bytes:
    if size == 4:
        props = struct.pack("<HHBBBBI", 0, 32, 23, 8, 0, 23, 127)
        sign = 31
    else:
        props = struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023)
        sign = 63
    return bytes([0x11, 0x20, sign, 0]) + struct.pack("<I", size) + props


def _dt_fixed_string(n: int) -> bytes:
    return bytes([0x13, 0, 0, 0]) + struct.pack("<I", n)


def _dt_vlen_string() -> bytes:
    return bytes([0x19, 0x01, 0, 0]) + struct.pack("<I", 16) + _dt_int(1, False)


_NP_TYPES = {
    np.dtype(np.uint8): lambda: _dt_int(1, False), np.dtype(np.uint16): lambda: _dt_int(2, False),
    np.dtype(np.uint32): lambda: _dt_int(4, False), np.dtype(np.uint64): lambda: _dt_int(8, False),
    np.dtype(np.int32): lambda: _dt_int(4, True), np.dtype(np.int64): lambda: _dt_int(8, True),
    np.dtype(np.float32): lambda: _dt_float(4), np.dtype(np.float64): lambda: _dt_float(8),
}


def _dspace(shape) -> bytes:
    shape = tuple(shape)
    return struct.pack("<BBBB4x", 1, len(shape), 0, 0) + b"".join(struct.pack("<Q", d) for d in shape)


class _File:
    def __init__(self):
        self.buf = bytearray(96)          # superblock, patched at the end
        self.gheap = None                 # [(index, bytes)] of the open global heap

    def put(self, data: bytes, align: int = 8) -> int:
        self.buf += b"\0" * (-len(self.buf) % align)
        addr = len(self.buf)
        self.buf += data
        return addr

    # --------------------------------------------------------- messages
    def header(self, msgs) -> int:
        body = b"".join(struct.pack("<HHB3x", t, len(_pad8(d)), 0) + _pad8(d) for t, d in msgs)
        return self.put(struct.pack("<BBHII", 1, 0, len(msgs), 1, len(body)) + b"\0" * 4 + body)

    @staticmethod
    def attr(name: str, value) -> bytes:
        if isinstance(value, str):
            raw = value.encode()
            dt, ds, data = _dt_fixed_string(max(1, len(raw))), _dspace(()), raw or b"\0"
        else:
            arr = np.asarray(value)
            dt = _NP_TYPES[arr.dtype]()
            ds = _dspace(arr.shape)
            data = arr.tobytes()
        nm = name.encode() + b"\0"
        return (struct.pack("<BBHHH", 1, 0, len(nm), len(dt), len(ds)) + _pad8(nm) + _pad8(dt) +
                _pad8(ds) + data)

    def dataset(self, arr: np.ndarray, attrs=None) -> int:
        arr = np.ascontiguousarray(arr)
        data_addr = self.put(arr.tobytes()) if arr.size else UNDEF
        msgs = [(0x0001, _dspace(arr.shape)), (0x0003, _NP_TYPES[arr.dtype]()),
                (0x0008, struct.pack("<BBQQ", 3, 1, data_addr, arr.nbytes))]
        msgs += [(0x000C, self.attr(k, v)) for k, v in (attrs or {}).items()]
        return self.header(msgs)

    def string_dataset(self, strings) -> int:
        """Variable-length strings in one global heap collection."""
        elems = b""
        payload = []
        for i, s in enumerate(strings, start=1):
            raw = s.encode()
            payload.append((i, raw))
        coll_body = b"".join(struct.pack("<HH4xQ", i, 1, len(raw)) + _pad8(raw) for i, raw in payload)
        size = max(4096, 16 + len(coll_body) + 16)
        free = size - 16 - len(coll_body)
        coll = b"GCOL" + bytes([1, 0, 0, 0]) + struct.pack("<Q", size) + coll_body
        coll += struct.pack("<HH4xQ", 0, 0, free) + b"\0" * (free - 16)
        coll_addr = self.put(coll)
        for i, raw in payload:
            elems += struct.pack("<IQI", len(raw), coll_addr, i)
        data_addr = self.put(elems) if elems else UNDEF
        msgs = [(0x0001, _dspace((len(strings),))), (0x0003, _dt_vlen_string()),
                (0x0008, struct.pack("<BBQQ", 3, 1, data_addr, len(elems)))]
        return self.header(msgs)

    def group(self, children: dict, attrs=None):
        """children: name -> (object header address, is_group, btree, heap).
        Returns (header address, btree address, heap address)."""
        names = sorted(children)
        heap_data = bytearray(8)          # offset 0: the empty name
        offs = {}
        for n in names:
            offs[n] = len(heap_data)
            heap_data += _pad8(n.encode() + b"\0")
        heap_data_addr = self.put(bytes(heap_data))
        heap_addr = self.put(b"HEAP" + bytes([0, 0, 0, 0]) +
                             struct.pack("<QQQ", len(heap_data), UNDEF, heap_data_addr))
        snods = []
        per = 2 * LEAF_K
        for c in range(0, max(1, len(names)), per):
            chunk = names[c:c + per]
            ents = b""
            for n in chunk:
                oh, is_group, bt, hp = children[n]
                scratch = struct.pack("<QQ", bt, hp) if is_group else b"\0" * 16
                ents += struct.pack("<QQII", offs[n], oh, 1 if is_group else 0, 0) + scratch
            ents += b"\0" * (40 * (per - len(chunk)))
            snods.append((self.put(b"SNOD" + bytes([1, 0]) + struct.pack("<H", len(chunk)) + ents),
                          chunk[-1] if chunk else ""))
        assert len(snods) <= 2 * INTERNAL_K, "too many links for one B-tree node"
        node = b"TREE" + bytes([0, 0]) + struct.pack("<HQQ", len(snods), UNDEF, UNDEF)
        node += struct.pack("<Q", 0)
        for addr, last in snods:
            node += struct.pack("<QQ", addr, offs.get(last, 0))
        node += b"\0" * (32 + 32 * INTERNAL_K - len(node))   # full node: 2K+1 keys, 2K children
        btree_addr = self.put(node)
        msgs = [(0x0011, struct.pack("<QQ", btree_addr, heap_addr))]
        msgs += [(0x000C, self.attr(k, v)) for k, v in (attrs or {}).items()]
        return self.header(msgs), btree_addr, heap_addr

    def finish(self, root) -> bytes:
        oh, bt, hp = root
        sb = b"\x89HDF\r\n\x1a\n" + bytes([0, 0, 0, 0, 0, 8, 8, 0])
        sb += struct.pack("<HHI", LEAF_K, INTERNAL_K, 0)
        sb += struct.pack("<QQQQ", 0, UNDEF, len(self.buf), UNDEF)
        sb += struct.pack("<QQII", 0, oh, 1, 0) + struct.pack("<QQ", bt, hp)
        assert len(sb) == 96
        self.buf[:96] = sb
        return bytes(self.buf)


def write_sketch_db(path: str, names, words: np.ndarray, kmers, sketchsize64: int,
                    lengths=None, base_freq=None, bbits: int = 14, random: dict | None = None,
                    codon_phased: bool = False):
    """words: uint64 [n_samples, n_kmers, sketchsize64 * bbits] (reference word layout).
    random: optional dict(k_min, k_max, use_rc, table: {name: cluster},
    matches: {k: CxC float}, centroids: Cx4 float)."""
    f = _File()
    kmers = [int(k) for k in kmers]
    words = np.ascontiguousarray(words, dtype=np.uint64)
    sketches = {}
    for i, name in enumerate(names):
        kids = {}
        for ki, k in enumerate(kmers):
            oh = f.dataset(words[i, ki], {"kmer-size": np.int32(k)})
            kids[str(k)] = (oh, False, 0, 0)
        attrs = {
            "sketchsize64": np.uint64(sketchsize64), "bbits": np.uint64(bbits),
            "length": np.uint64(3_000_000 if lengths is None else lengths[i]),
            "missing_bases": np.uint64(0), "reads": np.uint8(0),
            "base_freq": np.asarray([0.25] * 4 if base_freq is None else base_freq[i], np.float64),
            "kmers": np.asarray(kmers, np.int32),
        }
        oh, bt, hp = f.group(kids, attrs)
        sketches[name] = (oh, True, bt, hp)
    top = {}
    oh, bt, hp = f.group(sketches, {"sketch_version": "b200-test",
                                    "codon_phased": np.uint8(codon_phased),
                                    "reverse_complement": np.uint8(1)})
    top["sketches"] = (oh, True, bt, hp)
    if random is not None:
        rk = {}
        tnames = list(random["table"])
        rk["table_keys"] = (f.string_dataset(tnames), False, 0, 0)
        rk["table_values"] = (f.dataset(np.asarray([random["table"][n] for n in tnames], np.uint16)),
                              False, 0, 0)
        ks = sorted(random["matches"])
        mats = [np.asarray(random["matches"][k], np.float32) for k in ks]
        C = mats[0].shape[0]
        rk["matches_keys"] = (f.dataset(np.asarray(ks, np.uint64)), False, 0, 0)
        rk["matches_values"] = (f.dataset(np.concatenate([m.ravel() for m in mats]),
                                          {"dims": np.asarray([C, C, len(ks)], np.uint64)}),
                                False, 0, 0)
        cen = np.asarray(random["centroids"], np.float32)
        rk["centroids"] = (f.dataset(cen.ravel(), {"dims": np.asarray(cen.shape, np.uint64)}),
                           False, 0, 0)
        oh, bt, hp = f.group(rk, {"k_min": np.uint32(random["k_min"]),
                                  "k_max": np.uint32(random["k_max"]),
                                  "use_rc": np.uint8(random.get("use_rc", 1))})
        top["random"] = (oh, True, bt, hp)
    root = f.group(top)
    with open(path, "wb") as fh:
        fh.write(f.finish(root))
