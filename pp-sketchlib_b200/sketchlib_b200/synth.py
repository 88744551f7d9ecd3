"""Seeded synthetic sketch populations (bin-level tree generator).

A population is a tree over samples: parent[s] < s, -1 for roots.  Along the
branch into sample s a core divergence c ~ U(0, c_max) and an accessory
fraction a ~ U(0, a_max) are drawn; at k-mer length k each 14-bit bin value is
inherited from the parent, or resampled uniformly with probability
1 - (1 - c)^k (1 - a).  The probabilities are stored as uint32 thresholds
(p * 2^32) for the counter-based generator in the library (sk_synth_host /
sk_synth_device), which turns (seed, sample, k, bin) into bits identically on
the CPU and the GPU.

Sequences for the sketcher (`genomes`): a seeded population of whole genomes
on a random recursive tree, base by base.

Shapes used by the benchmarks and tests:
  random_tree          a random recursive tree (parents uniform over earlier samples)
  clade_tree           n_clades clades with log-normal sizes under one root
  query_population     queries hanging off reference samples, with a fraction
                       of novel clades that attach to the root instead
"""
from __future__ import annotations

import numpy as np

DEFAULT_KMERS = list(range(15, 31, 2))     # k = 15, 17, ..., 29 (8 lengths)


def thresholds(c: np.ndarray, a: np.ndarray, kmers) -> np.ndarray:
    k = np.asarray(kmers, dtype=np.float64)[None, :]
    p = 1.0 - (1.0 - c[:, None]) ** k * (1.0 - a[:, None])
    t = np.floor(p * 2.0 ** 32)
    return np.clip(t, 0, 2 ** 32 - 1).astype(np.uint32)


def random_tree(n: int, kmers=DEFAULT_KMERS, seed: int = 0x5EED0002, c_max: float = 0.03,
                a_max: float = 0.2):
    rng = np.random.default_rng(seed)
    parent = np.empty(n, dtype=np.int32)
    parent[0] = -1
    if n > 1:
        parent[1:] = (rng.random(n - 1) * np.arange(1, n)).astype(np.int32)
    c = rng.uniform(0.0, c_max, n)
    a = rng.uniform(0.0, a_max, n)
    return parent, thresholds(c, a, kmers)


def clade_tree(n: int, n_clades: int = 200, kmers=DEFAULT_KMERS, seed: int = 0x5EED0003,
               c_max: float = 0.03, a_max: float = 0.2, sigma: float = 1.0):
    """One root, n_clades clade founders under it, clade sizes log-normal."""
    rng = np.random.default_rng(seed)
    n_clades = max(1, min(n_clades, n - 1))
    w = rng.lognormal(0.0, sigma, n_clades)
    sizes = np.maximum(1, np.floor(w / w.sum() * (n - 1))).astype(np.int64)
    while sizes.sum() < n - 1:
        sizes[rng.integers(n_clades)] += 1
    while sizes.sum() > n - 1:
        i = int(np.argmax(sizes))
        sizes[i] -= 1
    parent = np.empty(n, dtype=np.int32)
    parent[0] = -1
    s = 1
    for size in sizes:
        founder = s
        parent[founder] = 0
        for m in range(1, int(size)):
            parent[founder + m] = founder + int(rng.integers(0, m))
        s += int(size)
    c = rng.uniform(0.0, c_max, n)
    a = rng.uniform(0.0, a_max, n)
    return parent, thresholds(c, a, kmers)


def query_population(ref_parent: np.ndarray, ref_thresh: np.ndarray, n_queries: int,
                     novel_frac: float = 0.05, kmers=DEFAULT_KMERS, seed: int = 0x5EED0005,
                     c_max: float = 0.03, a_max: float = 0.2):
    """Appends n_queries samples to a reference tree: each query descends from a
    random reference sample, or (novel_frac of them) from the root via a fresh
    clade founder.  Returns the joint (parent, thresh) and the query indices."""
    rng = np.random.default_rng(seed)
    n_ref = len(ref_parent)
    parent = list(ref_parent.tolist())
    extra_c, extra_a = [], []
    q_idx = []
    for _ in range(n_queries):
        if rng.random() < novel_frac:
            parent.append(0)          # a novel clade founder under the root
            extra_c.append(rng.uniform(0.0, c_max)); extra_a.append(rng.uniform(0.0, a_max))
            founder = len(parent) - 1
            parent.append(founder)    # the query itself
        else:
            parent.append(int(rng.integers(0, n_ref)))
        extra_c.append(rng.uniform(0.0, c_max)); extra_a.append(rng.uniform(0.0, a_max))
        q_idx.append(len(parent) - 1)
    parent = np.asarray(parent, dtype=np.int32)
    th = np.concatenate([ref_thresh, thresholds(np.asarray(extra_c), np.asarray(extra_a), kmers)])
    return parent, th, np.asarray(q_idx, dtype=np.int64)


def genomes(n: int, length: int, seed: int = 0x5EED0001, gc: float = 0.38,
            snp_max: float = 0.004, acc_max: float = 0.03, segment: int = 5000) -> np.ndarray:
    """n genomes of `length` bases (uint8 ASCII, shape (n, length)): the root
    draws i.i.d. bases at the given GC content; genome g > 0 copies a uniformly
    chosen earlier genome, changes a fraction U(0, snp_max) of positions to
    another base (core SNPs) and replaces a fraction U(0, acc_max) of the
    sequence with fresh random segments of `segment` bases (accessory)."""
    rng = np.random.default_rng(seed)
    p = [(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2]
    letters = np.frombuffer(b"ACGT", np.uint8)
    code = np.zeros(256, np.uint8)
    code[letters] = np.arange(4, dtype=np.uint8)
    out = np.empty((n, length), np.uint8)
    out[0] = letters[rng.choice(4, length, p=p)]
    for g in range(1, n):
        out[g] = out[int(rng.integers(0, g))]
        snps = int(rng.uniform(0, snp_max) * length)
        pos = rng.integers(0, length, snps)
        out[g, pos] = letters[(code[out[g, pos]] + rng.integers(1, 4, snps)) % 4]
        for _ in range(int(rng.uniform(0, acc_max) * length / segment)):
            start = int(rng.integers(0, length - segment))
            out[g, start:start + segment] = letters[rng.choice(4, segment, p=p)]
    return out
