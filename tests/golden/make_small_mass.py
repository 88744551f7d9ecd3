"""Extracts the real sketches of the reference's GPU test databases.

pp-sketchlib's GPU check (test/gpu_test.py) compares CPU and GPU distances on
test/small_mass.h5 (6 samples) and test/small_mass_plus1.h5 (the same 6 plus
6925_1_55), sketched at k = 14, 17, 20, 23, 26, 29 with sketchsize64 = 156.
This script reads small_mass_plus1.h5 with the library's own HDF5 reader and
stores its sketches as tests/golden/small_mass_sketches.npz so the GPU tests
run on real bacterial sketches without the reference tree:

  names   (7,)              sample names, database order
  kmers   (6,)              k-mer lengths
  words   (7, 6, 2184) u64  sketches in the reference word layout
  length  (7,) u64          sequence lengths (database default where absent)
  n_small ()                samples belonging to small_mass.h5 (the first 6)

Usage: python tests/golden/make_small_mass.py [path/to/reference]  (default: $PP_SKETCHLIB_REF)
"""
import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "pp-sketchlib_b200"))
import pp_sketchlib  # noqa: E402

ref = Path(sys.argv[1] if len(sys.argv) > 1 else os.environ["PP_SKETCHLIB_REF"]) / "test"
kmers = [14, 17, 20, 23, 26, 29]
plus1 = pp_sketchlib._load_sketch_db(str(ref / "small_mass_plus1"), [], kmers)
small = pp_sketchlib._load_sketch_db(str(ref / "small_mass"), [], kmers)
assert plus1["names"][:len(small["names"])] == small["names"]
assert np.array_equal(plus1["words"][:len(small["names"])], small["words"])
dest = Path(__file__).with_name("small_mass_sketches.npz")
np.savez_compressed(dest, names=np.asarray(plus1["names"]), kmers=np.asarray(kmers, np.int32),
                    words=plus1["words"], length=np.asarray(plus1["length"], np.uint64),
                    n_small=np.int64(len(small["names"])))
print(f"wrote {dest}")
