"""Extracts the reference's golden vectors into tests/golden/ref_goldens.npz.

Reads the regression-test outputs that pp-sketchlib ships in its test/
directory (test/ppsketch_ref{,_phased}{,_jaccard,_raw_jaccard}.npy, checked by
test/test-dists.py:156-203) from a reference checkout and stores them as one
small fixture, so the oracle pins run without the reference tree:

  <name>_coreacc      float32 (378, 2)  core, accessory per pair
  <name>_jaccard      float32 (378, K)  random-corrected Jaccard per k
  <name>_raw_jaccard  float32 (378, K)  uncorrected Jaccard per k
  <name>_kmers        int32   (K,)      k-mer lengths of that database

for name in {unphased (k = 15,19,23,27; `sketch -k 15,29,4`, test/run_test.py:28),
             phased (k = 15,19,23,27,31; the CLI default -k 15,31,4)},
all at sketch size 10000 (sketchsize64 156).

Usage: python tests/golden/make_golden.py [path/to/reference]  (default: $PP_SKETCHLIB_REF)
"""
import os
import sys
from pathlib import Path

import numpy as np

ref = Path(sys.argv[1] if len(sys.argv) > 1 else os.environ["PP_SKETCHLIB_REF"]) / "test"
out = {}
for name, stem, kmers in [("unphased", "ppsketch_ref", [15, 19, 23, 27]),
                          ("phased", "ppsketch_ref_phased", [15, 19, 23, 27, 31])]:
    out[f"{name}_coreacc"] = np.load(ref / f"{stem}.npy").astype(np.float32)
    out[f"{name}_jaccard"] = np.load(ref / f"{stem}_jaccard.npy").astype(np.float32)
    out[f"{name}_raw_jaccard"] = np.load(ref / f"{stem}_raw_jaccard.npy").astype(np.float32)
    out[f"{name}_kmers"] = np.asarray(kmers, dtype=np.int32)
dest = Path(__file__).with_name("ref_goldens.npz")
np.savez_compressed(dest, **out)
print(f"wrote {dest}: " + ", ".join(f"{k}{v.shape}" for k, v in out.items()))
