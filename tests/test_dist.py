"""Multi-rank host logic on CPU (gloo, world size 2): key-shard routing with
per-rank tables gives, op for op, the results of one table replaying the
whole stream, and the max-over-ranks timing reduction."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from lslab_b200 import shard
from lslab_b200 import workload as W


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _stream(n=30_000, seed=3):
    rng = np.random.default_rng(seed)
    types = rng.choice([0, 1, 2], size=n, p=[0.6, 0.3, 0.1]).astype(np.uint8)
    keys = W.key_of_rank(seed, rng.integers(0, 4000, size=n))
    vals = W.splitmix64(seed + 1, 0, n)
    return types, keys, vals


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import OracleMap
        types, keys, vals = _stream()
        parts = shard.route(types, keys, vals, world)
        idx, t, k, v = parts[rank]
        res = OracleMap(8).mixed(t, k, v)
        gathered = [None] * world
        dist.all_gather_object(gathered, (idx, res))
        m = shard.max_over_ranks(float(rank + 1))
        shard.barrier()
        if rank == 0:
            q.put((gathered, m))
    finally:
        dist.destroy_process_group()


def test_routed_shards_equal_single_table_replay():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    gathered, m = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert m == float(world)
    from oracle import OracleMap
    types, keys, vals = _stream()
    want = OracleMap(8).mixed(types, keys, vals)
    got = shard.merge_results([g[0] for g in gathered], [g[1] for g in gathered], len(keys),
                              want.dtype)
    assert np.array_equal(got, want)
    assert all(len(g[0]) > 0 for g in gathered)


def test_shard_of_is_balanced_and_stable():
    keys = W.prefill_keys(5, 1 << 16)
    for world in (2, 4, 8):
        s = shard.shard_of(keys, world)
        assert s.min() == 0 and s.max() == world - 1
        counts = np.bincount(s, minlength=world)
        assert counts.min() > 0.9 * len(keys) / world
        assert np.array_equal(s, shard.shard_of(keys, world))


def test_table_hash_matches_fmix64_vector():
    # MurmurHash3 fmix64 of 1 (published finaliser constants)
    assert int(shard.table_hash(np.array([1], np.uint64))[0]) == 0xB456BCFC34C2CB2C
