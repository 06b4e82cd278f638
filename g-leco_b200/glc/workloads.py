"""Seeded synthetic columns with the shapes of the benchmark workloads.

The reference benchmarks on SOSD books/fb/wiki and generated linear/normal columns
(data/download_data.sh, data/generate.py), none of which ships with it; these generators
stand in for them with the sizes and value distributions the workloads name:

* ``plain_small``      1,048,576 int32, v[i] = 1000*i + U{0..255}, fixed partitions of 1024.
* ``piecewise_linear`` uint64 piecewise-linear: segment lengths ~ Poisson(50,000), slope per
                       segment U{1..10^6}, intercept jump U{0..2^40} from the previous
                       segment's end, additive noise U[0, 2^b) with b from {0,4,8,16,24}.
* ``timestamps``       int64 cumulative sums of exponential gaps (mean 1000) rounded to
                       integers, starting at 0.
* ``lookup_positions`` half uniform positions, half Zipf(s=1.1) over partitions (rank to
                       partition by a seeded permutation) with a uniform offset inside.
"""
from __future__ import annotations

import numpy as np


def plain_small(n: int = 1 << 20, seed: int = 42) -> np.ndarray:
    rng = np.random.default_rng(seed)
    i = np.arange(n, dtype=np.int64)
    return (1000 * i + rng.integers(0, 256, n)).astype(np.int32)


def piecewise_linear(n: int, seed: int = 42, mean_segment: int = 50_000) -> np.ndarray:
    rng = np.random.default_rng(seed)
    lens = []
    total = 0
    while total < n:
        k = max(1, int(rng.poisson(mean_segment)))
        k = min(k, n - total)
        lens.append(k)
        total += k
    lens = np.array(lens, np.int64)
    S = len(lens)
    slope = rng.integers(1, 1_000_001, S).astype(np.uint64)
    jump = rng.integers(0, 1 << 40, S, endpoint=True).astype(np.uint64)
    bsel = rng.choice(np.array([0, 4, 8, 16, 24]), S)
    seg_start = np.concatenate([[0], np.cumsum(lens)[:-1]])
    # intercept_k = end value of segment k-1 (without noise) + jump_k
    seg_span = slope * (lens.astype(np.uint64) - np.uint64(1))
    base = np.zeros(S, np.uint64)
    acc = np.uint64(0)
    for k in range(S):
        acc = acc + jump[k]
        base[k] = acc
        acc = acc + seg_span[k]
    seg_id = np.repeat(np.arange(S), lens)
    j = (np.arange(n, dtype=np.int64) - seg_start[seg_id]).astype(np.uint64)
    v = base[seg_id] + slope[seg_id] * j
    bits = bsel[seg_id]
    noise = (rng.integers(0, 1 << 24, n, dtype=np.int64).astype(np.uint64)
             & ((np.uint64(1) << bits.astype(np.uint64)) - np.uint64(1)))
    return (v + noise).astype(np.uint64)


def timestamps(n: int, seed: int = 42, mean_gap: float = 1000.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    gaps = np.rint(rng.exponential(mean_gap, n)).astype(np.int64)
    gaps[0] = 0
    return np.cumsum(gaps, dtype=np.int64)


def lookup_positions(n: int, q: int, partition_len: int, seed: int = 42, zipf_s: float = 1.1) -> np.ndarray:
    rng = np.random.default_rng(seed + 1)
    P = (n + partition_len - 1) // partition_len
    q_uni = q // 2
    q_zipf = q - q_uni
    uni = rng.integers(0, n, q_uni, dtype=np.int64)
    ranks = np.arange(1, P + 1, dtype=np.float64)
    w = ranks ** (-zipf_s)
    w /= w.sum()
    perm = rng.permutation(P)
    part = perm[rng.choice(P, q_zipf, p=w)]
    start = part.astype(np.int64) * partition_len
    plen = np.minimum(partition_len, n - start)
    off = (rng.random(q_zipf) * plen).astype(np.int64)
    zipf = start + off
    pos = np.concatenate([uni, zipf])
    return pos.astype(np.int32)
