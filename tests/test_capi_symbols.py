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
