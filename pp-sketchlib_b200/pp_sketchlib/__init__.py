"""Drop-in ``pp_sketchlib`` module backed by the B200 distance library.

The distance functions of the reference module -- queryDatabase,
querySelfSparse, jaccardDist, squareToLong, longToSquare, longToSquareMulti,
sparsifyDistsByThreshold -- and constructDatabase keep their names, arguments
and return types; sketching and distances run on the GPU through the
library's C ABI.  Put the directory that
holds this package (pp-sketchlib_b200/) on sys.path and ``import pp_sketchlib``.
"""
from ._pp_sketchlib import (  # noqa: F401
    HDF5Exception,
    _load_random,
    _load_sketch_db,
    _read_sequences,
    _save_sketch_db,
    addRandom,
    constructDatabase,
    jaccardDist,
    longToSquare,
    longToSquareMulti,
    queryDatabase,
    querySelfSparse,
    sketchVersion,
    sparsifyDists,
    sparsifyDistsByThreshold,
    squareToLong,
    version,
)
