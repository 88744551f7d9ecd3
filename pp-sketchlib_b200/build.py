"""Build recipe for the B200 distance library (sm_100a) and its Python module.

Outputs, all in-tree so they travel with the repository snapshot:
  pp-sketchlib_b200/sketchlib_b200/libsketchlib_b200.so   C ABI + CUDA kernels
  pp-sketchlib_b200/pp_sketchlib/_pp_sketchlib*.so        pybind11 drop-in module

Run as ``python pp-sketchlib_b200/build.py`` (or through ``__graft_entry__.build``).
Each target is rebuilt only when one of its sources is newer than it.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
LIB = PKG / "sketchlib_b200" / "libsketchlib_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

CUDA_SOURCES = ["dist_kernel.cu", "aux_kernels.cu", "probe_kernels.cu", "capi.cu", "batch.cu",
                "serve.cu", "noalloc.cu", "query_db.cu", "sketch.cu"]


def _stale(target: Path, sources) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(s).stat().st_mtime > t for s in sources)


def _run(cmd):
    print(" ".join(str(c) for c in cmd), flush=True)
    subprocess.run([str(c) for c in cmd], check=True)


def build_library(force: bool = False) -> Path:
    sources = [CSRC / s for s in CUDA_SOURCES if (CSRC / s).exists()]
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    if not force and not _stale(LIB, sources + headers):
        return LIB
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    objs = []
    for src in sources:
        obj = objdir / (src.stem + ".o")
        if force or _stale(obj, [src] + headers):
            _run([NVCC, "-std=c++17", *ARCH, "-O3", "-lineinfo", "-Xcompiler", "-fPIC",
                  "-Xcompiler", "-O3", "-I", CSRC, "-I", INCLUDE, "-c", src, "-o", obj])
        objs.append(obj)
    _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs, "-lpthread"])
    return LIB


def build_module(force: bool = False) -> Path | None:
    src = CSRC / "pp_sketchlib_module.cpp"
    if not src.exists():
        return None
    try:
        import pybind11
    except ImportError:  # pragma: no cover - pybind11 ships with the image
        print("pybind11 missing: Python module not built", file=sys.stderr)
        return None
    suffix = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    out = PKG / "pp_sketchlib" / ("_pp_sketchlib" + suffix)
    deps = [src, LIB] + list(CSRC.glob("host_*.h")) + list(CSRC.glob("host_*.cpp")) + list(INCLUDE.glob("*.h"))
    if not force and not _stale(out, deps):
        return out
    host_srcs = sorted(CSRC.glob("host_*.cpp"))
    _run(["g++", "-std=c++17", "-O3", "-fPIC", "-shared", "-fvisibility=hidden",
          "-I", pybind11.get_include(), "-I", sysconfig.get_paths()["include"],
          "-I", INCLUDE, "-I", CSRC, src, *host_srcs, "-o", out,
          "-L", LIB.parent, "-lsketchlib_b200", "-Wl,-rpath,$ORIGIN/../sketchlib_b200",
          "-lpthread", "-lz"])
    return out


def main() -> None:
    force = "--force" in sys.argv
    build_library(force)
    build_module(force)


if __name__ == "__main__":
    main()
