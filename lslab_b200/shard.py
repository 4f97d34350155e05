"""Multi-GPU sharding of the map: one independent table per rank.

The path partitions by key: a key belongs to rank `shard_of(key, world)`
(high bits of the table hash, so the choice is independent of the bucket bits
each rank's table uses).  Ops on different keys commute, so running each
rank's ops in their original relative order on its own table gives, op for op,
the results of one table running the whole stream in index order.  There is
no data-path collective: routing happens where the ops are produced, and the
ranks only meet for timing (barrier, max over ranks).

The benchmark uses independent per-rank streams (weak scaling); `route` and
`merge_results` serve callers with one global stream.
"""
from __future__ import annotations

import numpy as np

_M1 = np.uint64(0xff51afd7ed558ccd)
_M2 = np.uint64(0xc4ceb9fe1a85ec53)


def table_hash(keys: np.ndarray) -> np.ndarray:
    """The tables' key hash (MurmurHash3 fmix64) for uint64 keys, on the host."""
    k = np.asarray(keys, np.uint64)
    with np.errstate(over="ignore"):
        k = k ^ (k >> np.uint64(33))
        k = k * _M1
        k = k ^ (k >> np.uint64(33))
        k = k * _M2
        return k ^ (k >> np.uint64(33))


def shard_of(keys: np.ndarray, world: int) -> np.ndarray:
    """Owning rank of each key: the top 16 hash bits times world, over 2^16."""
    top = (table_hash(keys) >> np.uint64(48)).astype(np.uint64)
    return ((top * np.uint64(world)) >> np.uint64(16)).astype(np.int64)


def route(types: np.ndarray, keys: np.ndarray, vals: np.ndarray | None, world: int):
    """Split one op stream by owning rank, keeping each rank's ops in their
    original order.  Returns, per rank, (op indices, types, keys, vals)."""
    owner = shard_of(keys, world)
    parts = []
    for r in range(world):
        idx = np.nonzero(owner == r)[0]
        parts.append((idx, types[idx], keys[idx], None if vals is None else vals[idx]))
    return parts


def merge_results(parts_idx, parts_out, n: int, dtype) -> np.ndarray:
    """Inverse of route for per-op results."""
    out = np.empty(n, dtype)
    for idx, res in zip(parts_idx, parts_out):
        out[idx] = res
    return out


def rank_seed(seed: int, rank: int) -> int:
    """Seed of rank `rank`'s independent stream in the weak-scaling benchmark."""
    return seed + 1000 * rank


def max_over_ranks(x: float) -> float:
    """Max of a host float over all ranks (identity without a process group).
    The reduction tensor lives on the backend's device (CUDA for nccl)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return x
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
