"""The benchmark's printed line (CPU only): one short JSON line with the
contract's keys and every section's headline numbers."""
import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))

import bench  # noqa: E402


def _record():
    parity = {"pairs": 10, "jaccard_max_vs_f64": 0.0, "well_conditioned": 9,
              "core": {"max_vs_f64": 0.0, "p99.9_vs_f64": 0.0, "max_vs_f32": 1.0e-5,
                       "p99.9_vs_f32": 1e-6, "above_1e-5_vs_f32": 0,
                       "max_vs_f32_well_conditioned": 1e-6},
              "accessory": {"max_vs_f64": 0.0, "p99.9_vs_f64": 0.0, "max_vs_f32": 1.0e-4,
                            "p99.9_vs_f32": 1e-5, "above_1e-5_vs_f32": 1,
                            "max_vs_f32_well_conditioned": 4e-6}}
    q = {"requests": 1000, "rate_hz": 5.0, "value": 1.0e7, "p50_ms": 22.123456, "p99_ms": 45.0,
         "max_ms": 60.0, "slices": 900, "slices_shared": 3, "queries_per_request": 100,
         "p99_under_50ms": True, "unit": "distances/s"}
    return {
        "metric": bench.METRIC, "value": 4.0e8, "unit": bench.UNIT, "n_gpus": 1, "steps": 20,
        "warmup": 3, "ms_per_step": 20.7891234, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": 67.0, "dtype": "u32", "data": "synthetic", "config": bench.workload_config(),
        "tile_config": "auto", "gpu_launches": 20, "clocks": {"sm_mhz": 1965.0},
        "cpu_baseline": {"value": 8e5, "unit": bench.UNIT, "cores": 16, "kind": "reference",
                         "sample": "rows"},
        "roofline": {"bound": "alu", "achieved": 14.1, "peak": 18.5, "unit": "T LOP3/s",
                     "frac": 0.7634567, "traffic": 4.4e9, "dram_gbs": 214.0, "popc_frac": 0.2,
                     "peak_source": "probe", "algorithmic": "x", "dram_frac_of_copy_peak": 0.03},
        "e2e": {"value": 3.4e8, "unit": bench.UNIT, "h2d_bytes_per_step": 1,
                "d2h_bytes_per_step": 1, "matches_resident_result": True, "steps": 5,
                "link_gbs": {"h2d": 55.0, "d2h": 55.0, "note": "x"}, "call": "x",
                "unpipelined": {"value": 2e8, "call": "x"}},
        "e2e_dropin": {"value": 1.1e8, "unit": bench.UNIT, "ms": 75.0, "steps": 3, "call": "x",
                       "file_bytes": 1, "result_shape": [1, 2]},
        "batched": {"value": 6.8e8, "lop3_frac": 0.7, "ms_per_batch": 113.0, "unit": bench.UNIT,
                    "plain_sequential": {"value": 5e8, "ms": 1.0, "launches": 40},
                    "pair_for_pair_equal_to_plain": True, "workload": "x", "pairs": 1,
                    "tile_config": 1, "work_items": 1, "timing": "x"},
        "serving": {"mixed": {**q, "p99_ms_le_128": 45.0, "n_le_128": 78,
                              "alone_vs_mixed_equal": True}, "q100": q,
                    "q100_sweep": [q, q], "q100_server": {"slots": 2, "slice_queries": 256}},
        "large": {"value": 4.5e8, "lop3_frac": 0.85, "knn": {"ms": 1130.0, "k": 10}},
        "sketch": {"value": 2.9e11, "unit": "k-mers/s", "e2e": {"value": 2.5e11},
                   "cpu_baseline": {"value": 1.4e9},
                   "reads": {"value": 183.0, "unit": "samples/s", "samples": 16,
                             "cpu_baseline": {"value": 1.1}}},
        "parity": {"samples4096": parity, "genomes": parity},
    }


def test_compact_line_is_short_and_complete():
    line = bench.compact_line(_record())
    text = json.dumps(line)
    assert len(text) < 4000
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "gpu_launches", "clocks", "cpu_baseline", "roofline", "e2e"):
        assert key in line, key
    for key in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert key in line["roofline"]
    assert line["e2e"]["h2d_bytes_per_step"] == 1
    assert line["serving"]["q100"]["p99_under_50ms"] is True
    assert line["parity"]["genomes"]["acc_above_1e-5_f32"] == 1
    assert line["roofline"]["frac"] == 0.763457 and line["ms_per_step"] == 20.7891
    assert line["config"] == bench.workload_config()
