#!/usr/bin/env python
"""Throughput of pp-sketchlib's all-vs-all core/accessory distance path on B200.

Workload (one "step"): the plain all-vs-all of 4,096 bin-level synthetic
samples (seeded random tree, k = 15, 17, ..., 29, sketchsize64 = 156 x 14 bit
planes, i.e. 8 k-mer lengths x 10,000 bins): 8,386,560 pairs written as float32
core/accessory in long form.  Inputs (573 MB of sketches) are larger than L2.

Arms:
  default            our CUDA path; `value` is device-timed with inputs resident
                     in HBM, `e2e` goes through the C ABI with pinned host
                     buffers (upload + pack + distances + result copy per step)
  --impl reference   the reference's CPU path (oracle/_ref: the reference's own
                     calc_intersize inside the query_db OpenMP loop) on this
                     host's cores, on bounded row samples of the same workload

Multi-GPU (torchrun): every rank runs its own replica of the workload (the path
has no exchange step); value = pairs of all ranks / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "pp-sketchlib_b200"))

METRIC = ("distances/sec @ 8 k × 10k bins (plain vs batched) on 1 B200; "
          "p50/p99 query latency")
UNIT = "distances/s"
N_SAMPLES = 4096
KMERS = list(range(15, 31, 2))
S64 = 156
BBITS = 14
SEED = 0x5EED0002
LOP3_PER_PAIR = len(KMERS) * 2 * S64 * BBITS        # one LOP3 per 32 bins per plane
POPC_PER_PAIR = len(KMERS) * 2 * S64
PUBLISHED_GPU = 6.0e6   # README.md:137,140 -- RTX 2080 Ti, 8 k x 10,000 bins
PROFILE_SUMMARY = ROOT / "profiles" / "dist_items_kernel_4096.md"


def n_pairs(n: int) -> int:
    return n * (n - 1) // 2


def workload_config():
    """The workload both arms report (identical dicts: per-arm details such as
    thread counts and tile shapes sit outside `config`)."""
    return {
        "workload": "plain all-vs-all, 4,096 bin-level synthetic samples (seeded random tree), "
                    "8 k-mer lengths x 10,000 bins (sketchsize64 156 x 14 planes), float32 "
                    "core/accessory long form",
        "n_samples": N_SAMPLES, "kmers": KMERS, "sketchsize64": S64, "bbits": BBITS,
        "pairs": n_pairs(N_SAMPLES), "seed": SEED,
        "l2": "inputs larger than L2 (573 MB of packed sketches vs 126 MB L2)",
    }


# ------------------------------------------------------------------ ranks

def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def init_dist(world: int, backend: str = "nccl"):
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))


def barrier(world: int, device=None):
    if world > 1:
        import torch.distributed as dist
        if device is not None and dist.get_backend() == "nccl":
            dist.barrier(device_ids=[device])
        else:
            dist.barrier()


def reduce_max(value: float, world: int, device: str = "cpu") -> float:
    """Max of a float over ranks (identity for one rank)."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ----------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi clock / throttle samples every 200 ms while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in getattr(self, "lines", []):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# -------------------------------------------------------------- baselines

def synth_module():
    """The numpy tree generator (pp-sketchlib_b200/sketchlib_b200/synth.py),
    loaded from its file alone: importing it through its package would load
    the library under test, which the reference arm must not map."""
    import importlib.util
    path = ROOT / "pp-sketchlib_b200" / "sketchlib_b200" / "synth.py"
    spec = importlib.util.spec_from_file_location("_bench_synth", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def reference_inputs(threads: int):
    """The workload's sketches, built by the oracle's restatement of the
    generator (bit-identical to the library's, tests/test_synth.py)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    synth = synth_module()
    parent, thresh = synth.random_tree(N_SAMPLES, kmers=KMERS, seed=SEED)
    return oracle.synth_words(parent, thresh, S64, SEED, threads=threads)


def cpu_reference_rate(target_s: float = 15.0, threads: int | None = None):
    """The reference's CPU path (oracle/_ref) on a bounded row sample of the
    workload; falls back to the oracle port when _ref was not built.  Uses
    nothing from the library under test."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import numpy as np
    import oracle
    threads = threads or os.cpu_count() or 1
    words = reference_inputs(threads)
    out = np.zeros((n_pairs(N_SAMPLES), 2), np.float32)
    if oracle.ref_available():
        kind = "reference"
        ref = oracle.RefQueryDb()
        prep = ref.prepare(words, KMERS, S64)

        def run(r0, r1):
            return ref.run_rows(prep, r0, r1, out, threads)
    else:
        kind = "port"

        def run(r0, r1):
            return oracle.dists_self_rows(words, KMERS, S64, r0, r1, out, threads)
    return kind, threads, run, words


def sample_rate(run, target_s: float):
    """Runs row blocks of the all-vs-all until ~target_s of CPU work is done."""
    row, pairs, elapsed, rows_per = 0, 0, 0.0, 2
    while elapsed < target_s and row < N_SAMPLES - 1:
        r1 = min(N_SAMPLES - 1, row + rows_per)
        t0 = time.perf_counter()
        done = run(row, r1)
        dt = time.perf_counter() - t0
        pairs += done
        elapsed += dt
        row = r1
        if dt < target_s / 8:
            rows_per *= 2
    return pairs, elapsed, row


def reference_gpu_rate(words, launches: int):
    """The reference's own GPU kernel (`calculate_dists`, src/gpu/dist.cu:164-317,
    compiled for sm_100a from the reference sources into oracle/_ref) on the
    full workload: inputs resident, one launch per step, CUDA events around
    each launch, launch shape from the reference's getBlockSize."""
    import torch
    if not torch.cuda.is_available():
        return None
    import oracle
    if not oracle.ref_gpu_available():
        return {"unavailable": "oracle/_ref/libref_gpu.so not built (needs the reference sources)"}
    _, ms = oracle.RefGpuKernel().self_dists(words, KMERS, S64, warmup=1, launches=launches,
                                             want_out=False)
    return {"value": n_pairs(N_SAMPLES) / (ms / 1e3), "unit": UNIT, "ms_per_launch": ms,
            "launches": launches,
            "kernel": "reference calculate_dists (src/gpu/dist.cu:164-317) built for sm_100a",
            "timing": "CUDA events per launch, sketches resident in the reference's "
                      "sample-minor layout, NoAdjust table"}


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    kind, threads, run, words = cpu_reference_rate()
    # A step is a block of consecutive rows: at least 16 per thread, so the
    # loop's dynamic schedule (5 rows per chunk) keeps every thread busy, and
    # about 1.5 s of work at the rate all threads reach on such a block.
    rows_per_step = min(N_SAMPLES // 4, 16 * threads)
    t0 = time.perf_counter()
    pairs = run(0, rows_per_step)
    rate = pairs / (time.perf_counter() - t0)
    while rows_per_step * 2 <= N_SAMPLES // 4 and rate * 1.5 > (N_SAMPLES - 1) * rows_per_step * 2:
        rows_per_step *= 2
    total_pairs, total_t, row = 0, 0.0, 0
    for step in range(args.warmup + args.steps):
        r0 = row % (N_SAMPLES - rows_per_step)
        t0 = time.perf_counter()
        done = run(r0, r0 + rows_per_step)
        dt = time.perf_counter() - t0
        row += rows_per_step
        if step >= args.warmup:
            total_pairs += done
            total_t += dt
    value = total_pairs / total_t
    sample = (f"{rows_per_step} consecutive all-vs-all rows of the 4,096-sample workload per step "
              f"({total_pairs} pairs over {args.steps} steps)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total_t / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded bin-level tree)",
        "config": workload_config(),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_ref_gpu:
        ref_gpu = reference_gpu_rate(words, max(1, min(args.steps, 5)))
        if ref_gpu is not None:
            line["reference_gpu_kernel"] = ref_gpu
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- our arm

def measured_hbm_gbs():
    """The pool's measured copy bandwidth (GB/s) from MEASURED_PEAKS.json, or None."""
    try:
        return float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return None


def profiled_traffic():
    """DRAM bytes per launch of the distance kernel from the committed ncu
    summary (line `dram_bytes_per_launch: N`), or None."""
    try:
        m = re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", PROFILE_SUMMARY.read_text())
        return float(m.group(1)) if m else None
    except OSError:
        return None


# ------------------------------------------------------------- sketching

SKETCH_GENOMES, SKETCH_LEN, SKETCH_SEED = 64, 2_500_000, 0x5EED0001
SKETCH_PROFILE = ROOT / "profiles" / "sketch_kernel_64_genomes.md"


# ALU-pipe instructions one canonical k-mer step of the sketch kernel needs, on
# 32-bit lanes, counted from its source (csrc/sketch.cu, roll_chunk and the
# emitter): forward split rotation and table XOR 7, reverse 7, canonical
# minimum (64-bit compare, two selects) 4, table-index and base-code
# extraction 2, run-length and window tests 7, reduction mod 2^61 - 1 10,
# exact bin (64-bit remainder test and increment; its multiplies run on the
# FMA pipe) 5, bin-minimum test 2.  The ALU utilisation ncu reports (70%)
# implies about 42 executed per k-mer.
SKETCH_ALU_OPS_PER_KMER = 44


def profiled_alu_pct():
    """ALU-pipe utilisation of the sketch kernel from the committed ncu
    summary (line `alu_pipe_pct: N`), or None."""
    try:
        m = re.search(r"alu_pipe_pct:\s*([0-9.]+)", SKETCH_PROFILE.read_text())
        return float(m.group(1)) if m else None
    except OSError:
        return None


def run_sketch(ctx, dev, steps, warmup, cpu=True, alu_peak=None):
    """Sketching of 64 genomes of 2.5 Mb at k = 15..29 odd, sketchsize64 156
    (the CPU parity case's shape): device-resident bases through
    sk_sketch_device (`value`), pinned host bases through sk_sketch (`e2e`),
    and the reference's own CPU sketcher on this host's cores."""
    import torch
    from sketchlib_b200 import capi, synth
    g = synth.genomes(SKETCH_GENOMES, SKETCH_LEN, seed=SKETCH_SEED)
    n, L = g.shape
    off = np.arange(n + 1, dtype=np.int64) * L
    ss = np.arange(n + 1, dtype=np.int64)
    kmers_step = sum(n * (L - k + 1) for k in KMERS)
    W = S64 * BBITS
    d_bases = torch.from_numpy(g.reshape(-1)).to(dev)
    d_words = torch.empty((n, len(KMERS), W), dtype=torch.int64, device=dev)

    def dev_step():
        capi.sketch_device(ctx, d_bases.data_ptr(), off, ss, KMERS, S64, d_words.data_ptr())

    for _ in range(warmup):
        dev_step()
    torch.cuda.synchronize(dev)
    call_ms = []
    for _ in range(steps):
        t0 = time.perf_counter()
        dev_step()      # returns after its stream has finished
        call_ms.append(1e3 * (time.perf_counter() - t0))
    sec = statistics.median(call_ms) / 1e3
    words_dev = d_words.cpu().numpy().view(np.uint64)

    pinned = torch.empty(n * L, dtype=torch.uint8).pin_memory()
    pinned.numpy()[:] = g.reshape(-1)
    host_words = torch.empty((n, len(KMERS), W), dtype=torch.int64).pin_memory().numpy().view(np.uint64)
    for _ in range(warmup):
        capi.sketch(ctx, pinned.numpy(), off, ss, KMERS, S64, words=host_words)
    e2e_ms = []
    for _ in range(steps):
        t0 = time.perf_counter()
        capi.sketch(ctx, pinned.numpy(), off, ss, KMERS, S64, words=host_words)
        e2e_ms.append(1e3 * (time.perf_counter() - t0))
    e2e_sec = statistics.median(e2e_ms) / 1e3
    out = {
        "workload": f"{n} genomes x {L:,} bases (i.i.d. bases at GC 0.38 on a random tree of "
                    "SNPs and 5 kb replacements), k = 15..29 odd, sketchsize64 156",
        "unit": "k-mers/s", "kmers_per_step": kmers_step,
        "value": kmers_step / sec, "ms_per_step": 1e3 * sec, "steps": steps,
        "timing": "host clock around each sk_sketch_device call (its planning, kernels and "
                  "the final synchronisation), median of the steps; bases resident in HBM",
        "e2e": {"value": kmers_step / e2e_sec, "unit": "k-mers/s", "ms_per_step": 1e3 * e2e_sec,
                "h2d_bytes_per_step": int(n * L),
                "d2h_bytes_per_step": int(host_words.nbytes + n * len(KMERS) * 9),
                "call": "sk_sketch from pinned host bases to pinned host sketches (upload in "
                        "sample chunks overlapped with hashing)",
                "matches_device_result": bool(np.array_equal(host_words, words_dev))},
        "roofline": {"bound": "alu", "alu_ops_per_kmer": SKETCH_ALU_OPS_PER_KMER,
                     "achieved": kmers_step / sec * SKETCH_ALU_OPS_PER_KMER / 1e12,
                     "peak": None if not alu_peak else alu_peak / 1e12, "unit": "T ALU op/s",
                     "frac": None if not alu_peak else
                     kmers_step / sec * SKETCH_ALU_OPS_PER_KMER / alu_peak,
                     "alu_pipe_pct_ncu": profiled_alu_pct(),
                     "source": str(SKETCH_PROFILE.relative_to(ROOT))},
    }
    if cpu:
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        if oracle.sketcher_available():
            kind = "reference"
            want = oracle.RefSketcher().sketch(g, KMERS, S64, threads=threads)
        else:
            kind = "port"
            want = oracle.sketch(g.reshape(-1), off, ss, KMERS, S64, True, threads=threads)[0]
        ct = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": kmers_step / ct, "unit": "k-mers/s", "cores": threads,
                               "kind": kind, "sample": f"the whole workload ({n} genomes, "
                                                       f"{ct:.2f} s)"}
        out["matches_cpu_sketcher"] = bool(np.array_equal(want, words_dev))
        # distances of the genomes (the CPU-runnable case) against the oracle
        gdb = capi.Database(ctx, words_dev, KMERS, S64)
        jac = capi.dists_dense(ctx, gdb, out_mode=capi.OUT_JACCARD)
        ca = capi.dists_dense(ctx, gdb)
        gdb.close()
        want_j, f64, f32 = oracle.dists_multi(want, KMERS, S64)
        out["genomes_parity"] = parity_stats(jac, want_j, ca, f64, f32)
        out["genomes_parity"]["sample"] = (f"all {n * (n - 1) // 2} pairs of the {n} genomes, "
                                           "sketched by the reference's sketcher")
    out["reads"] = run_sketch_reads(ctx, steps, warmup, cpu)
    return out


def read_set(rng):
    """133,333 reads of 150 bp: 10x coverage of a 2 Mb genome, 1% errors."""
    G, cov, RL = 2_000_000, 10, 150
    genome = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, G)]
    n_reads = cov * G // RL
    starts = rng.integers(0, G - RL, n_reads)
    reads = genome[starts[:, None] + np.arange(RL)[None, :]]
    err = rng.random(reads.shape) < 0.01
    reads[err] = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, int(err.sum()))]
    return reads


def run_sketch_reads(ctx, steps, warmup, cpu, n_samples=None):
    """A batch of read sets, each a 2 Mb genome at 10x coverage of 150 bp reads
    with 1% errors (20 Mbases), sketched with min_count = 3 (exact k-mer
    counts): one sample per host core, as the reference sketches one sample
    per thread.  The GPU sketches the whole batch in one sk_sketch call; the
    reference's CPU sketcher (exact = true, the same reads as FASTQ) runs the
    samples on that many threads."""
    import tempfile
    from concurrent.futures import ThreadPoolExecutor
    from sketchlib_b200 import capi
    cores = os.cpu_count() or 1
    n = n_samples or cores
    rng = np.random.default_rng(SKETCH_SEED + 1)
    reads = read_set(rng)
    n_reads, RL = reads.shape
    one = reads.reshape(-1)
    bases = np.tile(one, n)
    off = np.arange(n * n_reads + 1, dtype=np.int64) * RL
    ss = np.arange(n + 1, dtype=np.int64) * n_reads
    for _ in range(warmup):
        words, _, _ = capi.sketch(ctx, bases, off, ss, KMERS, S64, min_count=3)
    ms = []
    for _ in range(steps):
        t0 = time.perf_counter()
        words, _, _ = capi.sketch(ctx, bases, off, ss, KMERS, S64, min_count=3)
        ms.append(1e3 * (time.perf_counter() - t0))
    sec = statistics.median(ms) / 1e3
    out = {"workload": f"{n} read sets of {n_reads:,} reads x {RL} bp (10x of a 2 Mb genome, "
                       "1% errors), k = 15..29 odd, sketchsize64 156, min_count 3 (exact counts)",
           "samples": n, "bases": int(bases.size), "value": n / sec, "unit": "samples/s",
           "ms": 1e3 * sec,
           "call": "one sk_sketch call from host memory (per k: the hashes grouped by range, "
                   "each group counted in shared memory, then the bins)"}
    if cpu:
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle
        if oracle.sketcher_available():
            rs = oracle.RefSketcher()
            with tempfile.TemporaryDirectory() as tmp:
                fq = Path(tmp) / "reads.fq"
                q = b"\n+\n" + b"I" * RL + b"\n"
                with open(fq, "wb") as f:
                    for r in reads:
                        f.write(b"@r\n" + r.tobytes() + q)
                t0 = time.perf_counter()
                with ThreadPoolExecutor(cores) as pool:
                    res = list(pool.map(lambda _: rs.sketch_file(fq, KMERS, S64, True, 3, True),
                                        range(n)))
                ct = time.perf_counter() - t0
            out["cpu_baseline"] = {"value": n / ct, "unit": "samples/s", "cores": cores,
                                   "kind": "reference", "seconds": ct,
                                   "sample": f"the same {n} read sets as FASTQ, one per thread: "
                                             "the reference's SeqBuf + sketch() with exact "
                                             "counting"}
            out["matches_cpu_sketcher"] = bool(all(np.array_equal(r[0], words[i])
                                                   for i, r in enumerate(res)))
    return out


# ------------------------------------------------------- batched (config 4)

BATCH_SEED = 0x5EED0004


def batched_jobs(rng):
    """40 databases: N log-uniform in [50, 8000], 4-14 odd k from 13..39,
    sketch_size from {1024, 4096, 10000, 20000} (sketchsize64 = round(size/64)),
    half all-vs-all, half a 10% query slice against the rest."""
    jobs = []
    for _ in range(40):
        n = int(round(np.exp(rng.uniform(np.log(50), np.log(8000)))))
        K = int(rng.integers(4, 15))
        kmers = sorted(int(k) for k in rng.choice(np.arange(13, 40, 2), K, replace=False))
        s64 = int(round(int(rng.choice([1024, 4096, 10000, 20000])) / 64))
        self_ = bool(rng.random() < 0.5)
        jobs.append(dict(n=n, kmers=kmers, s64=s64, self=self_))
    return jobs


def run_batched(ctx, dev, lop3_peak, repeats=3, autotune=False):
    import torch
    from sketchlib_b200 import capi, synth
    rng = np.random.default_rng(BATCH_SEED)
    specs = batched_jobs(rng)
    made, lop3_total, pairs_total = [], 0, 0
    for j, sp in enumerate(specs):
        parent, thresh = synth.random_tree(sp["n"], kmers=sp["kmers"], seed=BATCH_SEED + j)
        words = torch.empty(sp["n"] * len(sp["kmers"]) * sp["s64"] * BBITS, dtype=torch.int64,
                            device=dev)
        capi.synth_device(ctx, parent, thresh, sp["s64"], seed=BATCH_SEED + j,
                          d_words=words.data_ptr())
        wps = len(sp["kmers"]) * sp["s64"] * BBITS
        if sp["self"]:
            ref = capi.Database(ctx, words.data_ptr(), sp["kmers"], sp["s64"], n_samples=sp["n"])
            qry = None
        else:
            nq = max(1, sp["n"] // 10)
            qry = capi.Database(ctx, words.data_ptr(), sp["kmers"], sp["s64"], n_samples=nq)
            ref = capi.Database(ctx, words.data_ptr() + nq * wps * 8, sp["kmers"], sp["s64"],
                                n_samples=sp["n"] - nq)
        del words
        rows = capi.dists_rows(ref, qry)
        out = torch.empty((max(rows, 1), 2), dtype=torch.float32, device=dev)
        made.append((ref, qry, None, capi.OUT_CORE_ACC, out))
        pairs_total += rows
        lop3_total += rows * len(sp["kmers"]) * 2 * sp["s64"] * BBITS
    batch = capi.Batch(ctx, [(r, q, rnd, m, o.data_ptr()) for r, q, rnd, m, o in made],
                       autotune=autotune)
    info = batch.info()
    batch.run()                      # warm-up
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(repeats):
        batch.launch()
    ctx.synchronize()
    batched_s = (time.perf_counter() - t0) / repeats
    ref_out = [o.clone() for *_, o in made]
    # the same jobs one plain call after another (each its own launch)
    capi_calls = 0
    ctx.synchronize()
    t0 = time.perf_counter()
    for r, q, rnd, m, o in made:
        capi.dists_dense(ctx, r, q, rnd, out_mode=m, out=o.data_ptr())
        capi_calls += 1
    ctx.synchronize()
    plain_s = time.perf_counter() - t0
    same = all(torch.equal(a, o) for a, (*_, o) in zip(ref_out, made))
    batch.close()
    for r, q, *_ in made:
        r.close()
        if q is not None:
            q.close()
    return {
        "workload": "40 databases, N log-uniform [50, 8000], 4-14 odd k in 13..39, sketchsize64 "
                    "in {16, 64, 156, 312}, half all-vs-all / half 10% queries vs the rest, "
                    "one graph-captured persistent launch",
        "value": pairs_total / batched_s, "unit": UNIT, "pairs": pairs_total,
        "ms_per_batch": 1e3 * batched_s, "lop3_frac": lop3_total / batched_s / lop3_peak,
        "tile_config": info["tile_config"], "work_items": info["n_items"],
        "plain_sequential": {"value": pairs_total / plain_s, "ms": 1e3 * plain_s,
                             "launches": capi_calls},
        "pair_for_pair_equal_to_plain": bool(same), "timing": "host clock around graph replays"
                                                              " (device work dominates)",
    }


# ------------------------------------------------------- serving (config 5)

SERVE_SEED = 0x5EED0005
SERVE_KMERS = list(range(15, 34, 2))
SERVE_N_REF, SERVE_POOL = 50_000, 4_000
# The 100-query run: 5 requests/s, a step below the highest rate whose p99
# stayed under 50 ms in a sweep of 1,000-request streams (4, 5, 6, 7 /s:
# p99 40.4, 40.6, 49.1, 40.7 ms; p50 22.8 ms), on a server of 2 slots x
# 256-query slices (which beat 4 x 128 at every rate).
Q100_RATE = 5.0
Q100_SLOTS, Q100_SLICE = 2, 256


def serving_setup(ctx, dev):
    """50,000 resident references (10 k-mer lengths, 15..33, sketchsize64 156)
    and a pool of 4,000 query sketches from the same tree, 5% from novel
    clades; the reference database is resident in HBM."""
    import torch
    from sketchlib_b200 import capi, synth
    kmers = SERVE_KMERS
    rp, rt = synth.clade_tree(SERVE_N_REF, n_clades=200, kmers=kmers, seed=SERVE_SEED)
    parent, thresh, qidx = synth.query_population(rp, rt, SERVE_POOL, novel_frac=0.05,
                                                  kmers=kmers, seed=SERVE_SEED + 1)
    n_all = len(parent)
    wps = len(kmers) * S64 * BBITS
    words = torch.empty(n_all * wps, dtype=torch.int64, device=dev)
    capi.synth_device(ctx, parent, thresh, S64, seed=SERVE_SEED, d_words=words.data_ptr())
    ref = capi.Database(ctx, words.data_ptr(), kmers, S64, n_samples=SERVE_N_REF)
    # the query pool in page-locked memory, as a server's receive buffers
    # would be: the server uploads such requests without staging them
    pool = torch.empty((SERVE_POOL, wps), dtype=torch.int64).pin_memory()
    pool.copy_(words.view(n_all, wps)[torch.as_tensor(qidx, device=dev)])
    qwords = pool.numpy().view(np.uint64).reshape(SERVE_POOL, len(kmers), S64 * BBITS)
    del words
    return ref, qwords, pool


def serve_stream(server, qwords, sizes, starts, gaps, check=()):
    """Submits requests as a Poisson stream (inter-arrival gaps in seconds)
    from a separate thread; returns latencies (s), the makespan and the
    results of the requests listed in `check`."""
    import threading
    n = len(sizes)
    tickets = [None] * n
    t_begin = time.perf_counter()

    def arrivals():
        t_next = time.perf_counter()
        for i in range(n):
            t_next += gaps[i]
            d = t_next - time.perf_counter()
            if d > 0:
                time.sleep(d)
            tickets[i] = server.submit(qwords[starts[i]:starts[i] + sizes[i]])

    th = threading.Thread(target=arrivals)
    th.start()
    th.join()
    lat = np.zeros(n)
    kept = {}
    for i in range(n):
        server.wait(tickets[i], timeout=600)
        idx, dist, _, lat[i] = server.result(tickets[i])
        if i in check:
            kept[i] = (idx, dist)
    return lat, time.perf_counter() - t_begin, kept


def pct_ms(a, q):
    return round(float(np.percentile(a, q) * 1e3), 2) if len(a) else None


def run_serving(ctx, dev, n_requests=120, rate_hz=10.0, q100_requests=1000, q100_rate=Q100_RATE,
                sweep=(), q100_slots=Q100_SLOTS, q100_slice=Q100_SLICE, sweep_requests=400):
    """(a) the mixed stream: batches of 1..2000 queries (log-uniform) at
    rate_hz; (b) q100_requests batches of exactly 100 queries at q100_rate;
    (c) optionally the same 100-query stream at each rate of `sweep`
    (sweep_requests each).  The 100-query runs use their own server with
    q100_slots slots of q100_slice queries.  Every query is scored against all
    references, top-5 kNN returned."""
    from sketchlib_b200 import capi
    ref, qwords, _pool = serving_setup(ctx, dev)
    n_ref, pool = SERVE_N_REF, SERVE_POOL
    server = capi.Server(ctx, ref, slots=4, slice_queries=128, kNN=5, large_slice_queries=64)
    t = server.submit(qwords[:64])       # warm-up request
    server.wait(t)
    server.result(t)
    out = {"references": n_ref, "kmers": len(SERVE_KMERS), "kNN": 5, "slots": 4,
           "slice_queries": 128, "large_slice_queries": 64}

    # (a) mixed sizes
    rng = np.random.default_rng(SERVE_SEED + 2)
    sizes = np.exp(rng.uniform(0, np.log(2000), n_requests)).astype(int).clip(1, 2000)
    starts = rng.integers(0, pool - sizes + 1)
    gaps = rng.exponential(1.0 / rate_hz, n_requests)
    check = [i for i in range(n_requests) if sizes[i] <= 500][:8]
    info0 = server.info()
    lat, makespan, mixed = serve_stream(server, qwords, sizes, starts, gaps, check)
    info1 = server.info()
    alone_equal = True
    for i in check:                      # the same requests again, alone on an idle server
        t = server.submit(qwords[starts[i]:starts[i] + sizes[i]])
        server.wait(t, timeout=600)
        idx, dist, _, _ = server.result(t)
        alone_equal &= bool(np.array_equal(idx, mixed[i][0]) and np.array_equal(dist, mixed[i][1]))
    one = sizes <= 128
    near100 = (sizes > 64) & (sizes <= 128)
    out["mixed"] = {
        "requests": n_requests, "rate_hz": rate_hz, "queries": int(sizes.sum()),
        "value": int(sizes.sum()) * n_ref / makespan, "unit": UNIT,
        "p50_ms": pct_ms(lat, 50), "p99_ms": pct_ms(lat, 99), "max_ms": pct_ms(lat, 100),
        "n_le_128": int(one.sum()), "p99_ms_le_128": pct_ms(lat[one], 99),
        "n_65_128": int(near100.sum()), "p99_ms_65_128": pct_ms(lat[near100], 99),
        "slices": info1["slices"] - info0["slices"],
        "slices_shared": info1["slices_shared"] - info0["slices_shared"],
        "alone_vs_mixed_equal": alone_equal, "alone_vs_mixed_checked": len(check)}

    server.close()
    server = capi.Server(ctx, ref, slots=q100_slots, slice_queries=q100_slice, kNN=5)
    t = server.submit(qwords[:100])      # warm-up request
    server.wait(t)
    server.result(t)
    out["q100_server"] = {"slots": q100_slots, "slice_queries": q100_slice}

    def q100(n_req, rate, seed):
        r = np.random.default_rng(seed)
        sz = np.full(n_req, 100)
        st = r.integers(0, pool - 100 + 1, n_req)
        gp = r.exponential(1.0 / rate, n_req)
        i0 = server.info()
        lt, mk, _ = serve_stream(server, qwords, sz, st, gp)
        i1 = server.info()
        return {"requests": n_req, "rate_hz": rate, "queries_per_request": 100,
                "value": n_req * 100 * n_ref / mk, "unit": UNIT,
                "p50_ms": pct_ms(lt, 50), "p99_ms": pct_ms(lt, 99), "max_ms": pct_ms(lt, 100),
                "slices": i1["slices"] - i0["slices"],
                "slices_shared": i1["slices_shared"] - i0["slices_shared"]}

    if q100_requests:
        out["q100"] = q100(q100_requests, q100_rate, SERVE_SEED + 3)
        out["q100"]["p99_under_50ms"] = out["q100"]["p99_ms"] < 50.0
    if sweep:
        out["q100_sweep"] = [q100(sweep_requests, float(r), SERVE_SEED + 4 + k)
                             for k, r in enumerate(sweep)]
    server.close()
    ref.close()
    return out


# ------------------------------------------------------------ large (config 3)

LARGE_SEED = 0x5EED0003
LARGE_N = 31_610


def run_large(ctx, dev, lop3_peak, launches=2, knn=10):
    """31,610 samples (200 clades, log-normal sizes), K = 8, sketchsize64 156:
    499,580,245 pairs written to a 4.0 GB device long form, then the
    kNN = 10 sparse graph (316,100 entries) through sk_dists_knn."""
    import torch
    from sketchlib_b200 import capi, synth
    n = LARGE_N
    parent, thresh = synth.clade_tree(n, n_clades=200, kmers=KMERS, seed=LARGE_SEED)
    words = torch.empty(n * len(KMERS) * S64 * BBITS, dtype=torch.int64, device=dev)
    capi.synth_device(ctx, parent, thresh, S64, seed=LARGE_SEED, d_words=words.data_ptr())
    db = capi.Database(ctx, words.data_ptr(), KMERS, S64, n_samples=n)
    del words
    pairs = n_pairs(n)
    out = torch.empty((pairs, 2), dtype=torch.float32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    ctx.set_stream(stream.cuda_stream)
    capi.dists_dense(ctx, db, out=out.data_ptr())          # warm-up
    ctx.synchronize()
    times = []
    with torch.cuda.stream(stream):
        for _ in range(launches):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            capi.dists_dense(ctx, db, out=out.data_ptr())
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
    finite = bool(torch.isfinite(out).all().item())
    del out
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    capi.dists_knn(ctx, db, knn, dist_col=0)        # first call grows the scratch buffers
    knn_first_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    i, j, d = capi.dists_knn(ctx, db, knn, dist_col=0)
    knn_s = time.perf_counter() - t0
    db.close()
    sec = sum(times) / len(times)
    return {
        "workload": "31,610 samples, 200 clades (log-normal sizes), 8 k x 10k bins, "
                    "float32 long form in HBM (4.0 GB) + kNN = 10 sparse graph",
        "n_samples": n, "pairs": pairs, "value": pairs / sec, "unit": UNIT,
        "ms_per_launch": 1e3 * sec, "launches": launches,
        "lop3_frac": pairs * LOP3_PER_PAIR / sec / lop3_peak,
        "knn": {"k": knn, "entries": int(len(i)), "ms": 1e3 * knn_s,
                "first_call_ms": 1e3 * knn_first_s,
                "timing": "host clock around a warm sk_dists_knn (distance kernel into a "
                          "2 GB column, top-k pass, D2H of the lists)"},
        "all_finite": finite,
    }


# ----------------------------------------------------------- parity, drop-in

WELL_CONDITIONED = 5e-6   # float-LDLT fit vs FP64 fit, both outputs


def parity_stats(jac_got, jac_want, ca_got, ca_f64, ca_f32):
    """Error of the CUDA path's outputs against the FP64 oracle and against the
    float-LDLT restatement of the reference's fit_slope; `well_conditioned`
    counts the pairs whose float fit agrees with the FP64 fit to 5e-6."""
    dj = np.abs(jac_got.astype(np.float64) - jac_want)
    d64 = np.abs(ca_got.astype(np.float64) - ca_f64)
    d32 = np.abs(ca_got.astype(np.float64) - ca_f32)
    well = (np.abs(ca_f32.astype(np.float64) - ca_f64) <= WELL_CONDITIONED).all(axis=1)
    out = {"pairs": int(ca_got.shape[0]), "jaccard_max_vs_f64": float(dj.max()),
           "well_conditioned": int(well.sum())}
    for c, name in enumerate(("core", "accessory")):
        out[name] = {"max_vs_f64": float(d64[:, c].max()),
                     "p99.9_vs_f64": float(np.quantile(d64[:, c], 0.999)),
                     "max_vs_f32": float(d32[:, c].max()),
                     "p99.9_vs_f32": float(np.quantile(d32[:, c], 0.999)),
                     "above_1e-5_vs_f32": int((d32[:, c] > 1e-5).sum()),
                     "max_vs_f32_well_conditioned": float(d32[well, c].max()) if well.any()
                     else 0.0}
    return out


def run_parity_rows(ctx, db, words, out_dev, rows=128):
    """The first `rows` rows of the all-vs-all (the longest rows) against the
    oracle: Jaccard, core and accessory, FP64 and float-LDLT fits."""
    from sketchlib_b200 import capi
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    n = words.shape[0]
    m = n * rows - rows * (rows + 1) // 2
    jac = capi.dists_dense(ctx, db, out_mode=capi.OUT_JACCARD)[:m]
    ca = out_dev[:m].cpu().numpy()
    t0 = time.perf_counter()
    want_j, f64, f32 = oracle.dists_multi(words, KMERS, S64, row_begin=0, row_end=rows)
    out = parity_stats(jac, want_j, ca, f64, f32)
    out["sample"] = f"all-vs-all rows 0..{rows - 1} ({m} pairs, oracle {time.perf_counter() - t0:.1f} s)"
    return out


def run_dropin(device, words, steps):
    """The reference-facing call end to end: pp_sketchlib.queryDatabase on an
    HDF5 sketch database of the 4,096 samples (written once, outside the timed
    region), self query with random_correct = True (equal-base correction, the
    reference's default without a /random group), use_gpu = True: read,
    flatten, upload, distances, and the numpy result."""
    import tempfile
    import pp_sketchlib
    n = words.shape[0]
    names = [f"sample{i:05d}" for i in range(n)]
    with tempfile.TemporaryDirectory() as tmp:
        db = str(Path(tmp) / "samples4096")
        pp_sketchlib._save_sketch_db(db, names, words, KMERS, S64, lengths=[2_500_000] * n)

        def call():
            return pp_sketchlib.queryDatabase(db, db, names, names, KMERS, random_correct=True,
                                              use_gpu=True, device_id=device)

        res = call()                      # warm-up (the module's context, scratch)
        ms = []
        for _ in range(steps):
            t0 = time.perf_counter()
            res = call()
            ms.append(1e3 * (time.perf_counter() - t0))
        fsize = Path(db + ".h5").stat().st_size
    sec = statistics.median(ms) / 1e3
    return {"value": n_pairs(n) / sec, "unit": UNIT, "ms": round(1e3 * sec, 2), "steps": steps,
            "file_bytes": int(fsize), "result_shape": list(res.shape),
            "call": "pp_sketchlib.queryDatabase(db, db, names, names, klist, use_gpu=True) from "
                    "an HDF5 file in the page cache (sketches read, uploaded, distances, numpy "
                    "result)"}


def rounded(x, digits=6):
    """Floats rounded to `digits` significant digits, recursively (the bench
    line stays one short line)."""
    if isinstance(x, float):
        return float(f"{x:.{digits}g}")
    if isinstance(x, dict):
        return {k: rounded(v, digits) for k, v in x.items()}
    if isinstance(x, list):
        return [rounded(v, digits) for v in x]
    return x


def run_ours(args, rank, world, local):
    import numpy as np
    import torch
    from sketchlib_b200 import capi, synth

    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    ctx = capi.Context(local)
    stream = torch.cuda.Stream(device=dev)
    ctx.set_stream(stream.cuda_stream)
    if args.tile_config:
        ctx.set_tile_config(args.tile_config)

    seed = SEED + rank
    parent, thresh = synth.random_tree(N_SAMPLES, kmers=KMERS, seed=seed)
    words_dev = torch.empty(N_SAMPLES * len(KMERS) * S64 * BBITS, dtype=torch.int64, device=dev)
    capi.synth_device(ctx, parent, thresh, S64, seed=seed, d_words=words_dev.data_ptr())
    db = capi.Database(ctx, words_dev.data_ptr(), KMERS, S64, n_samples=N_SAMPLES)
    pairs = n_pairs(N_SAMPLES)
    out = torch.empty((pairs, 2), dtype=torch.float32, device=dev)

    lop3_peak, popc_peak = capi.probe_alu_peak(ctx)

    # ---- device-timed, inputs resident in HBM
    for _ in range(args.warmup):
        capi.dists_dense(ctx, db, out=out.data_ptr())
    ctx.synchronize()
    barrier(world, local)
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with ClockSampler(local) as clocks:
        with torch.cuda.stream(stream):
            for s in range(args.steps):
                starts[s].record(stream)
                capi.dists_dense(ctx, db, out=out.data_ptr())
                ends[s].record(stream)
        ctx.synchronize()
        torch.cuda.synchronize()
    barrier(world, local)
    step_ms = [a.elapsed_time(b) for a, b in zip(starts, ends)]
    total_s = starts[0].elapsed_time(ends[-1]) / 1e3
    total_s = reduce_max(total_s, world, dev)
    value = pairs * args.steps * world / total_s
    launch_s = statistics.mean(step_ms) / 1e3

    # ---- end to end through the C ABI with pinned host buffers
    host_words = torch.empty(words_dev.numel(), dtype=torch.int64, pin_memory=True)
    host_words.copy_(words_dev.cpu())
    host_out = torch.empty((pairs, 2), dtype=torch.float32, pin_memory=True)
    hw = host_words.numpy().view(np.uint64).reshape(N_SAMPLES, len(KMERS), S64 * BBITS)
    ho = host_out.numpy()

    def e2e_step():
        # one sk_query_db call: chunked upload overlapped with the kernel
        capi.query_db(ctx, hw, KMERS, S64, out=ho)

    def e2e_step_unpipelined():
        # upload, then compute, then copy back (sk_db_create + sk_dists_dense)
        d = capi.Database(ctx, hw, KMERS, S64)
        capi.dists_dense(ctx, d, out=ho)
        d.close()

    def time_e2e(step, n):
        for _ in range(min(args.warmup, 3)):
            step()
        barrier(world, local)
        t0 = time.perf_counter()
        for _ in range(n):
            step()
        return reduce_max(time.perf_counter() - t0, world, dev)

    def link_gbs():
        """Plain pinned copies of this step's input (H2D) and output (D2H), GB/s."""
        dev_in = torch.empty_like(host_words, device=dev)
        dev_out = torch.empty_like(host_out, device=dev)
        rates = []
        for src, dst in ((host_words, dev_in), (dev_out, host_out)):
            dst.copy_(src, non_blocking=True)
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(3):
                dst.copy_(src, non_blocking=True)
            e1.record()
            e1.synchronize()
            rates.append(3 * src.numel() * src.element_size() / (e0.elapsed_time(e1) / 1e3) / 1e9)
        del dev_in, dev_out
        return rates

    h2d_gbs, d2h_gbs = link_gbs()
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    e2e_s = time_e2e(e2e_step, e2e_steps)
    e2e_value = pairs * world * e2e_steps / e2e_s
    # the e2e result must be the resident run's result
    ok = bool(torch.equal(host_out, out.cpu()))
    seq_s = time_e2e(e2e_step_unpipelined, e2e_steps)
    ok = ok and bool(torch.equal(host_out, out.cpu()))

    extra = {}
    if not args.skip_dropin:
        extra["e2e_dropin"] = run_dropin(local, hw, max(1, min(args.steps, 3)))
    if not args.skip_batched:
        extra["batched"] = run_batched(ctx, dev, lop3_peak, autotune=args.batch_autotune)
    if not args.skip_serving:
        sweep = [float(r) for r in args.serving_sweep.split(",")] if args.serving_sweep else ()
        extra["serving"] = run_serving(ctx, dev, q100_requests=args.q100_requests,
                                       q100_rate=args.q100_rate, sweep=sweep,
                                       q100_slots=args.q100_slots, q100_slice=args.q100_slice,
                                       sweep_requests=args.sweep_requests)
    if world == 1 and not args.skip_large:
        extra["large"] = run_large(ctx, dev, lop3_peak)
    if not args.skip_sketch:
        extra["sketch"] = run_sketch(ctx, dev, max(3, min(args.steps, 10)), max(1, args.warmup),
                                     cpu=rank == 0 and world == 1 and not args.no_cpu_baseline,
                                     alu_peak=lop3_peak)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        kind, threads, run, _ = cpu_reference_rate()
        cp, ct, rows = sample_rate(run, args.cpu_seconds)
        cpu = {"value": cp / ct, "unit": UNIT, "cores": threads, "kind": kind,
               "sample": f"rows 0..{rows - 1} of the 4,096-sample all-vs-all ({cp} pairs, "
                         f"{ct:.1f} s)"}
        # the oracle as the checker of this run's results (outside every timed region)
        extra["parity"] = {"samples4096": run_parity_rows(ctx, db, hw, out)}
        if "sketch" in extra and "genomes_parity" in extra["sketch"]:
            extra["parity"]["genomes"] = extra["sketch"].pop("genomes_parity")

    achieved = pairs * LOP3_PER_PAIR / launch_s
    traffic = profiled_traffic()
    hbm_peak = measured_hbm_gbs()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total_s / args.steps,
        "higher_is_better": True, "scaling": "weak",
        "vs_baseline": value / PUBLISHED_GPU,
        "dtype": "u32", "data": "synthetic (seeded bin-level tree, generated on device)",
        "config": workload_config(),
        "tile_config": args.tile_config or "auto",
        "vs_baseline_source": "reference README.md:137,140 GPU figure, 6.0e6 distances/s "
                              "(RTX 2080 Ti)",
        "roofline": {"bound": "alu", "achieved": achieved / 1e12, "peak": lop3_peak / 1e12,
                     "unit": "T LOP3/s", "frac": achieved / lop3_peak,
                     "traffic": traffic,
                     "dram_gbs": None if traffic is None else traffic / launch_s / 1e9,
                     "dram_frac_of_copy_peak": None if traffic is None or not hbm_peak
                                               else traffic / launch_s / 1e9 / hbm_peak,
                     "peak_source": "sk_probe_alu_peak, measured in this run (LOP3 chains on "
                                    "every SM); popc peak %.3g/s" % popc_peak,
                     "algorithmic": f"{LOP3_PER_PAIR} LOP3 + {POPC_PER_PAIR} POPC per pair x "
                                    f"{pairs} pairs per launch",
                     "popc_frac": pairs * POPC_PER_PAIR / launch_s / popc_peak},
        "e2e": {"value": e2e_value, "unit": UNIT,
                "h2d_bytes_per_step": int(host_words.numel() * 8),
                "d2h_bytes_per_step": int(host_out.numel() * 4),
                "steps": e2e_steps, "matches_resident_result": ok,
                "link_gbs": {"h2d": h2d_gbs, "d2h": d2h_gbs,
                             "note": "plain pinned copies of the step's input and output on "
                                     "this box; the upload alone takes "
                                     f"{host_words.numel() * 8 / h2d_gbs / 1e6:.1f} ms"},
                "call": "sk_query_db (upload in sample chunks on a copy stream, each chunk's "
                        "tiles computed while the next copies)",
                "unpipelined": {"value": pairs * world * e2e_steps / seq_s,
                                "call": "sk_db_create + sk_dists_dense"}},
        "gpu_launches": args.steps,
        "clocks": clocks.summary(),
        "kernel_ms": {"mean": statistics.mean(step_ms), "min": min(step_ms),
                      "max": max(step_ms)},
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    line.update(extra)
    if rank == 0:
        if args.details:
            Path(args.details).parent.mkdir(parents=True, exist_ok=True)
            Path(args.details).write_text(json.dumps(line, indent=1))
        print(json.dumps(compact_line(line)), flush=True)
    db.close()
    ctx.close()


def compact_line(line):
    """The bench line: the contract's keys and each section's headline numbers
    (the full record goes to --details)."""
    keep = ["metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
            "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
            "tile_config", "gpu_launches", "clocks", "cpu_baseline"]
    out = {k: line[k] for k in keep if k in line}
    rf = line["roofline"]
    out["roofline"] = {k: rf[k] for k in ("bound", "achieved", "peak", "unit", "frac", "traffic",
                                          "dram_gbs", "popc_frac")}
    e = line["e2e"]
    out["e2e"] = {k: e[k] for k in ("value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step",
                                    "matches_resident_result")}
    out["e2e"]["link_gbs"] = {k: e["link_gbs"][k] for k in ("h2d", "d2h")}
    if "e2e_dropin" in line:
        d = line["e2e_dropin"]
        out["e2e_dropin"] = {k: d[k] for k in ("value", "unit", "ms")}
    if "batched" in line:
        b = line["batched"]
        out["batched"] = {"value": b["value"], "lop3_frac": b["lop3_frac"],
                          "ms": b["ms_per_batch"], "plain_sequential": b["plain_sequential"]["value"],
                          "equal_to_plain": b["pair_for_pair_equal_to_plain"]}
    if "serving" in line:
        sv = line["serving"]
        out["serving"] = {}
        for key in ("mixed", "q100"):
            if key in sv:
                out["serving"][key] = {k: sv[key][k] for k in sv[key]
                                       if k in ("requests", "rate_hz", "value", "p50_ms", "p99_ms",
                                                "p99_ms_le_128", "n_le_128", "slices_shared",
                                                "alone_vs_mixed_equal", "p99_under_50ms")}
        if "q100_sweep" in sv:
            out["serving"]["q100_sweep"] = [[r["rate_hz"], r["p50_ms"], r["p99_ms"]]
                                            for r in sv["q100_sweep"]]
        if "q100_server" in sv:
            out["serving"]["q100_server"] = sv["q100_server"]
    if "large" in line:
        lg = line["large"]
        out["large"] = {"value": lg["value"], "lop3_frac": lg["lop3_frac"],
                        "knn_ms": lg["knn"]["ms"]}
    if "sketch" in line:
        sk = line["sketch"]
        out["sketch"] = {"value": sk["value"], "unit": sk["unit"], "e2e": sk["e2e"]["value"]}
        if sk.get("roofline", {}).get("frac") is not None:
            out["sketch"]["alu_frac"] = sk["roofline"]["frac"]
        if "cpu_baseline" in sk:
            out["sketch"]["cpu_baseline"] = sk["cpu_baseline"]["value"]
        rd = sk.get("reads", {})
        if rd:
            out["sketch"]["reads"] = {"value": rd["value"], "unit": rd["unit"],
                                      "samples": rd["samples"]}
            if "cpu_baseline" in rd:
                out["sketch"]["reads"]["cpu_baseline"] = rd["cpu_baseline"]["value"]
    if "parity" in line:
        out["parity"] = {}
        for key, p in line["parity"].items():
            out["parity"][key] = {"pairs": p["pairs"], "jaccard_max": p["jaccard_max_vs_f64"],
                                  "core_max_f64": p["core"]["max_vs_f64"],
                                  "acc_max_f64": p["accessory"]["max_vs_f64"],
                                  "core_max_f32": p["core"]["max_vs_f32"],
                                  "acc_max_f32": p["accessory"]["max_vs_f32"],
                                  "acc_above_1e-5_f32": p["accessory"]["above_1e-5_vs_f32"],
                                  "well_conditioned": p["well_conditioned"]}
    return rounded(out)


def run_profile_case(n: int, launches: int):
    """A small case for ncu: n samples, `launches` dense launches, nothing else."""
    import torch
    from sketchlib_b200 import capi, synth
    ctx = capi.Context(0)
    parent, thresh = synth.random_tree(n, kmers=KMERS, seed=SEED)
    words = torch.empty(n * len(KMERS) * S64 * BBITS, dtype=torch.int64, device="cuda")
    capi.synth_device(ctx, parent, thresh, S64, seed=SEED, d_words=words.data_ptr())
    db = capi.Database(ctx, words.data_ptr(), KMERS, S64, n_samples=n)
    out = torch.empty((n_pairs(n), 2), dtype=torch.float32, device="cuda")
    for _ in range(launches):
        capi.dists_dense(ctx, db, out=out.data_ptr())
    ctx.synchronize()
    print(json.dumps({"profile_case": n, "pairs": n_pairs(n), "launches": launches}))
    db.close()
    ctx.close()


def run_profile_sketch(n: int, launches: int):
    """A small sketching case for ncu: n genomes of 2.5 Mb from device memory,
    `launches` sk_sketch_device calls, nothing else."""
    import torch
    from sketchlib_b200 import capi, synth
    ctx = capi.Context(0)
    g = synth.genomes(n, SKETCH_LEN, seed=SKETCH_SEED)
    off = np.arange(n + 1, dtype=np.int64) * SKETCH_LEN
    ss = np.arange(n + 1, dtype=np.int64)
    d_bases = torch.from_numpy(g.reshape(-1)).cuda()
    d_words = torch.empty((n, len(KMERS), S64 * BBITS), dtype=torch.int64, device="cuda")
    for _ in range(launches):
        capi.sketch_device(ctx, d_bases.data_ptr(), off, ss, KMERS, S64, d_words.data_ptr())
    print(json.dumps({"profile_sketch": n, "launches": launches}))
    ctx.close()


def run_profile_sketch_reads(launches: int):
    """A small case for ncu: the bench's 20 Mbase read set through sk_sketch
    with min_count 3, `launches` times, nothing else."""
    from sketchlib_b200 import capi
    ctx = capi.Context(0)
    reads = read_set(np.random.default_rng(SKETCH_SEED + 1))
    n_reads, RL = reads.shape
    off = np.arange(n_reads + 1, dtype=np.int64) * RL
    ss = np.array([0, n_reads], np.int64)
    for _ in range(launches):
        capi.sketch(ctx, reads.reshape(-1), off, ss, KMERS, S64, min_count=3)
    print(json.dumps({"profile_sketch_reads": int(reads.size), "launches": launches}))
    ctx.close()


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--tile-config", type=int, default=0)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--skip-batched", action="store_true")
    ap.add_argument("--skip-serving", action="store_true")
    ap.add_argument("--skip-dropin", action="store_true",
                    help="skip timing pp_sketchlib.queryDatabase on an HDF5 database")
    ap.add_argument("--q100-requests", type=int, default=1000,
                    help="requests of exactly 100 queries in the serving run (0: none)")
    ap.add_argument("--q100-rate", type=float, default=Q100_RATE)
    ap.add_argument("--q100-slots", type=int, default=Q100_SLOTS)
    ap.add_argument("--q100-slice", type=int, default=Q100_SLICE)
    ap.add_argument("--sweep-requests", type=int, default=400)
    ap.add_argument("--serving-sweep", default="",
                    help="comma-separated arrival rates for 100-query streams of 400 requests")
    ap.add_argument("--details", default="",
                    help="also write the full record (every section) to this JSON file")
    ap.add_argument("--skip-sketch", action="store_true",
                    help="skip the sketching section (64 genomes x 2.5 Mb)")
    ap.add_argument("--batch-autotune", action="store_true",
                    help="let the batch time every tile shape at creation (outside the timed region)")
    ap.add_argument("--skip-large", action="store_true",
                    help="skip the 31,610-sample all-vs-all + kNN = 10 measurement")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="--impl reference: skip timing the reference's GPU kernel")
    ap.add_argument("--profile", type=int, default=0,
                    help="run only N-sample dense launches (a small case for ncu)")
    ap.add_argument("--profile-launches", type=int, default=2)
    ap.add_argument("--profile-sketch", type=int, default=0,
                    help="run only N genomes through sk_sketch_device (for ncu)")
    ap.add_argument("--profile-sketch-reads", action="store_true",
                    help="run only the 20 Mbase read set through sk_sketch (for ncu)")
    args = ap.parse_args()
    if args.profile_sketch:
        run_profile_sketch(args.profile_sketch, args.profile_launches)
        return
    if args.profile_sketch_reads:
        run_profile_sketch_reads(args.profile_launches)
        return
    if args.profile:
        run_profile_case(args.profile, args.profile_launches)
        return
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    init_dist(world)
    try:
        run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
