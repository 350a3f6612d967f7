"""Seeded synthetic workloads of the five benchmark configurations.

Every pair is generated by ``tsu_gen_batch`` (i.i.d. uniform ACGT pattern;
text = pattern with E = round(L * rate) edits, equal insertion and deletion
counts, the rest substitutions, at distinct uniform positions).  Lengths and
rates per pair come from numpy's PCG64 with a fixed seed, so every workload is
reproducible.  No public dataset is involved: these stand in for the shapes
the reference's artifact scripts (run_h100-a100.sh) generate.

  c1  10,000 x 150 bp, 2 %                       (CPU-runnable configuration)
  c2  1,000,000 x 1,000 bp, 5 %                  (plain GPU at scale)
  c3  20,000 x 10,000 bp, 15 %                   (long erroneous reads)
  c4  200,000 pairs, L log-uniform 100..20,000,  (batched uneven)
      rate uniform 1..15 % per pair
  c5  serving mixture per pair: 70 % 150 bp @ 1-3 %, 25 % U[1,5] kbp @ 5-10 %,
      5 % U[10,50] kbp @ 10-20 %; requests of U{1..256} pairs
"""
from __future__ import annotations

from typing import Tuple

import numpy as np

SEED = 0x5453554E414D49


def _rng(index: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(SEED + index))


def shape(name: str, n: int = 0) -> Tuple[np.ndarray, np.ndarray, int]:
    """(lengths int32[n], rates float64[n], generator seed) of a workload;
    n = 0 takes the configuration's own pair count."""
    if name == "c1":
        n = n or 10_000
        return np.full(n, 150, np.int32), np.full(n, 0.02), SEED + 0
    if name == "c2":
        n = n or 1_000_000
        return np.full(n, 1000, np.int32), np.full(n, 0.05), SEED + 1
    if name == "c3":
        n = n or 20_000
        return np.full(n, 10_000, np.int32), np.full(n, 0.15), SEED + 2
    if name == "c4":
        n = n or 200_000
        r = _rng(3)
        lengths = np.exp(r.uniform(np.log(100), np.log(20_000), n)).astype(np.int32)
        rates = r.uniform(0.01, 0.15, n)
        return lengths, rates, SEED + 3
    if name == "c5":
        n = n or 100_000
        r = _rng(4)
        u = r.uniform(0, 1, n)
        lengths = np.where(u < 0.70, 150, np.where(u < 0.95, r.integers(1000, 5001, n), r.integers(10_000, 50_001, n)))
        rates = np.where(u < 0.70, r.uniform(0.01, 0.03, n),
                         np.where(u < 0.95, r.uniform(0.05, 0.10, n), r.uniform(0.10, 0.20, n)))
        return lengths.astype(np.int32), rates, SEED + 4
    raise ValueError(f"unknown workload {name}")


def generate(name: str, n: int = 0, first: int = 0):
    """Concatenated buffers (pbuf, poff, plen, tbuf, toff, tlen) of a workload."""
    from . import gen_batch

    lengths, rates, seed = shape(name, n)
    return gen_batch(seed, lengths, rates, first=first)


def length_buckets(lengths: np.ndarray) -> np.ndarray:
    """floor(log2(L)) per pair: the buckets of the one-launch-per-uniform-batch
    (plain) form."""
    return np.floor(np.log2(np.maximum(lengths, 1))).astype(np.int32)


def c5_stream(n_requests: int, rate_per_s: float, index: int = 0, max_pairs: int = 256):
    """A serving stream: arrival times in seconds (Poisson process of
    rate_per_s, the first at 0) and request sizes (uniform 1..max_pairs
    pairs) of n_requests requests.  Pairs are drawn from the c5 mixture in
    order (request k takes the next sizes[k] pairs)."""
    r = _rng(5 + index)
    gaps = r.exponential(1.0 / rate_per_s, n_requests)
    arrivals = np.cumsum(gaps) - gaps[0]
    sizes = r.integers(1, max_pairs + 1, n_requests).astype(np.int64)
    return arrivals, sizes
