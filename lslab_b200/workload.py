"""Seeded synthetic workloads for the map/set hot path.

Every input (keys, op types, values) is a pure function of a seed and a
counter, so the CUDA path, the reference's kernels, the oracle and the host
replay all see bit-identical inputs.

* splitmix64: the counter form of Steele/Lea/Flood's SplitMix64 generator
  (state_i = seed + (i+1) * 0x9E3779B97F4A7C15, then the published 3-step
  xor-shift-multiply finaliser).  The finaliser is a bijection, so distinct
  counters give distinct keys.
* Zipf(theta) ranks over [0, N): the sampler of Gray et al., "Quickly
  Generating Billion-Record Synthetic Databases" (SIGMOD 1994); zeta(N, theta)
  is summed exactly for the first 2^20 terms and by Euler-Maclaurin beyond.
  Rank r maps to the r-th key of the prefill stream, so hot keys are
  unstructured 64-bit values.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
VALUE_XOR = 0x9E3779B97F4A7C15

OP_GET, OP_PUT, OP_REMOVE, OP_UPDATE = 0, 1, 2, 3
OP_CONTAINS, OP_INSERT = 0, 1

# stream offsets added to a workload's base seed
S_PREFILL, S_ABSENT, S_TYPES, S_ZIPF, S_VALUES, S_SIZES, S_ARRIVAL = 1, 2, 3, 4, 5, 6, 7


def splitmix64(seed: int, start: int, count: int) -> np.ndarray:
    """Outputs start .. start+count-1 of the SplitMix64 stream of `seed`."""
    with np.errstate(over="ignore"):
        x = np.arange(start + 1, start + count + 1, dtype=np.uint64) * GOLDEN
        x = x + np.uint64(seed & 0xFFFFFFFFFFFFFFFF)
        z = (x ^ (x >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def uniform01(seed: int, start: int, count: int) -> np.ndarray:
    """Doubles in [0, 1) from the top 53 bits of the stream."""
    return (splitmix64(seed, start, count) >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)


_ZETA: dict[tuple[int, float], float] = {}


def zeta(n: int, theta: float) -> float:
    key = (n, theta)
    if key in _ZETA:
        return _ZETA[key]
    m = min(n, 1 << 20)
    s = float(np.sum(np.arange(1, m + 1, dtype=np.float64) ** (-theta)))
    if n > m:
        f = lambda x: x ** (-theta)
        fp = lambda x: -theta * x ** (-theta - 1.0)
        s += (n ** (1.0 - theta) - m ** (1.0 - theta)) / (1.0 - theta)
        s += (f(n) - f(m)) / 2.0 + (fp(n) - fp(m)) / 12.0
    _ZETA[key] = s
    return s


def zipf_ranks(n_items: int, theta: float, seed: int, start: int, count: int) -> np.ndarray:
    """Zipf(theta) ranks in [0, n_items), rank 0 the most frequent (Gray et al. 1994)."""
    zn = zeta(n_items, theta)
    z2 = 1.0 + 0.5 ** theta
    alpha = 1.0 / (1.0 - theta)
    eta = (1.0 - (2.0 / n_items) ** (1.0 - theta)) / (1.0 - z2 / zn)
    u = uniform01(seed, start, count)
    uz = u * zn
    r = np.floor(n_items * np.power(eta * u - eta + 1.0, alpha))
    r = np.where(uz < 1.0, 0.0, np.where(uz < z2, 1.0, r))
    return np.clip(r, 0, n_items - 1).astype(np.int64)


def prefill_keys(seed: int, count: int, start: int = 0) -> np.ndarray:
    return splitmix64(seed + S_PREFILL, start, count)


def key_of_rank(seed: int, ranks: np.ndarray) -> np.ndarray:
    """Key of Zipf rank r = the r-th prefill key, computed from the counter."""
    with np.errstate(over="ignore"):
        x = (ranks.astype(np.uint64) + np.uint64(1)) * GOLDEN + np.uint64(seed + S_PREFILL)
        z = (x ^ (x >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def prefill_values(keys: np.ndarray) -> np.ndarray:
    return keys ^ np.uint64(VALUE_XOR)


def absent_keys(seed: int, count: int, present: np.ndarray | None = None,
                start: int = 0) -> np.ndarray:
    """Keys from a disjoint stream; any that collide with `present` are dropped."""
    k = splitmix64(seed + S_ABSENT, start, count)
    if present is not None and len(present):
        k = k[~np.isin(k, present)]
    return k


def type_sorted(types: np.ndarray, *arrays: np.ndarray):
    """Stable partition of a batch by op type (gets/contains, then puts/inserts,
    then removes): the order in which a per-op-type caller issues the batch."""
    order = np.argsort(types, kind="stable")
    return (types[order],) + tuple(a[order] for a in arrays)


# ---------------------------------------------------------------- configs
@dataclass
class MixedBatch:
    types: np.ndarray  # uint8
    keys: np.ndarray   # uint64 (map) / uint32 (set)
    vals: np.ndarray | None


def map_zipf_batch(seed: int, batch: int, n_ops: int, n_items: int, theta: float,
                   mix: tuple[float, ...], type_sort: bool = True) -> MixedBatch:
    """One batch of the map's mixed workload.  `mix` = (get, put[, remove])
    fractions; keys Zipf(theta) over the n_items prefill keys; put values
    uniform u64.  With type_sort the batch is issued gets, puts, removes."""
    start = batch * n_ops
    u = uniform01(seed + S_TYPES, start, n_ops)
    cum = np.cumsum(np.asarray(mix, dtype=np.float64))
    types = np.searchsorted(cum[:-1], u, side="right").astype(np.uint8)
    ranks = zipf_ranks(n_items, theta, seed + S_ZIPF, start, n_ops)
    keys = key_of_rank(seed, ranks)
    vals = splitmix64(seed + S_VALUES, start, n_ops)
    if type_sort:
        types, keys, vals = type_sorted(types, keys, vals)
    return MixedBatch(types, keys, vals)


def lognormal_sizes(seed: int, count: int, median: float, sigma: float, lo: int,
                    hi: int) -> np.ndarray:
    """Batch sizes: lognormal(median, sigma) clipped to [lo, hi] (Box-Muller
    on two uniform streams)."""
    u1 = uniform01(seed + S_SIZES, 0, count)
    u2 = uniform01(seed + S_SIZES, count, count)
    z = np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * math.pi * u2)
    s = np.exp(math.log(median) + sigma * z)
    return np.clip(np.rint(s), lo, hi).astype(np.int64)


def set_mixed_batch(seed: int, batch: int, n_ops: int, mix=(0.5, 0.4, 0.1),
                    type_sort: bool = True) -> MixedBatch:
    """Set workload batch: uniform u32 keys; mix = (contains, insert, remove)."""
    start = batch * n_ops
    u = uniform01(seed + S_TYPES, start, n_ops)
    cum = np.cumsum(np.asarray(mix, dtype=np.float64))
    types = np.searchsorted(cum[:-1], u, side="right").astype(np.uint8)
    keys = (splitmix64(seed + S_ZIPF, start, n_ops) >> np.uint64(32)).astype(np.uint32)
    if type_sort:
        types, keys = type_sorted(types, keys)
    return MixedBatch(types, keys, None)


def perm32(idx: np.ndarray) -> np.ndarray:
    """Distinct u32 keys: a bijective 32-bit mix of idx (odd multiplies and
    xor-shifts modulo 2^32), the same function the set sweep applies on the
    device."""
    x = np.asarray(idx).astype(np.uint64) & np.uint64(0xFFFFFFFF)
    m = np.uint64(0xFFFFFFFF)
    with np.errstate(over="ignore"):
        x = ((x ^ (x >> np.uint64(16))) * np.uint64(0x7FEB352D)) & m
        x = ((x ^ (x >> np.uint64(15))) * np.uint64(0x846CA68B)) & m
        x = x ^ (x >> np.uint64(16))
    return x.astype(np.uint32)


def set_prefill_keys(seed: int, count: int) -> np.ndarray:
    """Distinct uniform u32 keys for a set prefill (duplicates removed, so the
    count can come out slightly below `count`)."""
    k = (splitmix64(seed + S_PREFILL, 0, count) >> np.uint64(32)).astype(np.uint32)
    _, first = np.unique(k, return_index=True)
    return k[np.sort(first)]


def serving_pool(seed: int, count: int, max_ops: int = 4096, n_items: int = 1 << 28,
                 theta: float = 0.99, put_frac: float = 0.5):
    """A pool of serving requests: sizes uniform in [1, max_ops], ops get/put
    with probability 1 - put_frac / put_frac in arrival order, keys Zipf(theta)
    over n_items keys, put values uniform u64.  Returns (pool_off, pool_n,
    types, keys, vals) with each request's ops contiguous."""
    u = uniform01(seed + S_SIZES, 0, count)
    n = np.minimum((u * max_ops).astype(np.int64) + 1, max_ops).astype(np.uint32)
    off = np.concatenate([[0], np.cumsum(n.astype(np.uint64))[:-1]]).astype(np.uint64)
    total = int(n.astype(np.uint64).sum())
    types = (uniform01(seed + S_TYPES, 0, total) < put_frac).astype(np.uint8)
    keys = key_of_rank(seed, zipf_ranks(n_items, theta, seed + S_ZIPF, 0, total))
    vals = splitmix64(seed + S_VALUES, 0, total)
    return off, n, types, keys, vals
