"""The C ABI library loads on a machine without a GPU and exports every entry
point include/sketchlib_b200.h declares (no compute calls here)."""
import ctypes
import re

import pytest

from conftest import ROOT


def declared_symbols():
    text = (ROOT / "include" / "sketchlib_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sk_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("sk_ctx_create", "sk_db_create", "sk_dists_dense", "sk_dists_knn",
                 "sk_random_create", "sk_sparse_threshold", "sk_long_to_square"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from sketchlib_b200 import capi
    lib = ctypes.CDLL(str(capi.LIB_PATH))
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from sketchlib_b200 import capi
    bound = set(capi.exported_symbols()) | set(capi._OPTIONAL)
    missing = [n for n in declared_symbols() if n not in bound]
    assert not missing, missing


def test_no_device_needed_for_metadata():
    from sketchlib_b200 import capi
    assert capi.lib.sk_abi_version() == 1
    cfgs = capi.tile_configs()
    assert cfgs and all(c["tile_rows"] % c["tile_cols"] == 0 for c in cfgs)
    assert capi.lib.sk_tile_config_info(999, *([None] * 5)) != 0


def header_structs():
    """Field names, offsets and sizes of the header's plain structs, laid out
    with the x86-64 C rules (each field aligned to its size)."""
    text = (ROOT / "include" / "sketchlib_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    sizes = {"int32_t": 4, "uint32_t": 4, "int64_t": 8, "uint64_t": 8, "uint16_t": 2, "double": 8}
    out = {}
    for name, body in re.findall(r"typedef struct (\w+) \{(.*?)\} \1;", text, flags=re.S):
        fields, off = [], 0
        for typ, ptr, field in re.findall(r"(?:const\s+)?(\w+)\s*(\*?)\s*(\w+);", body):
            size = 8 if ptr else sizes[typ]
            off = (off + size - 1) // size * size
            fields.append((field, off))
            off += size
        align = max(8 if p else sizes[t] for t, p, _ in
                    re.findall(r"(?:const\s+)?(\w+)\s*(\*?)\s*(\w+);", body))
        out[name] = (fields, (off + align - 1) // align * align)
    return out


@pytest.mark.parametrize("c_name,py_name", [("sk_host_sketches", "HostSketches"),
                                            ("sk_job", "Job"),
                                            ("sk_server_params", "ServerParams")])
def test_ctypes_structs_match_header(c_name, py_name):
    """The Python binding's ctypes mirrors have the header's fields, in order,
    at the same offsets, and the same size."""
    from sketchlib_b200 import capi
    fields, size = header_structs()[c_name]
    cls = getattr(capi, py_name)
    assert [f for f, _ in fields] == [f[0] for f in cls._fields_]
    assert [o for _, o in fields] == [getattr(cls, f).offset for f, _ in fields]
    assert ctypes.sizeof(cls) == size
