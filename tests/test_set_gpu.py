"""GPU parity of the set against the oracle."""
from __future__ import annotations

import numpy as np
import pytest

from lslab_b200 import Set, OP_CONTAINS, OP_INSERT, OP_REMOVE
from lslab_b200 import workload as W
from oracle import OracleSet
from tests.util import dev, host

pytestmark = pytest.mark.gpu


def _bools(n, cuda):
    return cuda.full((n,), 7, dtype=cuda.uint8, device="cuda")


def test_contains_insert_remove_known_answer(cuda):
    """test/set_test.cu:40-81: keys 1..1024 on 2^10 buckets, 100 reps of
    insert -> contains all true -> remove -> contains all false (from rep 1 on
    every insert goes into a removed slot)."""
    s = Set(10)
    keys = dev(np.arange(1, 1025, dtype=np.uint32))
    r1, r2 = _bools(1024, cuda), _bools(1024, cuda)
    for rep in range(100):
        s.insert(keys, r1)
        s.contains(keys, r2)
        cuda.cuda.synchronize()
        assert (host(r1, np.uint8) == 1).all()
        assert (host(r2, np.uint8) == 1).all()
        s.remove(keys, r1)
        s.contains(keys, r2)
        cuda.cuda.synchronize()
        assert (host(r1, np.uint8) == 1).all()
        assert (host(r2, np.uint8) == 0).all()
    assert s.size() == 0
    assert s.status() == 0


@pytest.mark.parametrize("fused,split", [(False, 100), (True, 100), (True, 0)])
@pytest.mark.parametrize("window", [0, 2048])
def test_set_mixed_conflicts_vs_oracle(cuda, fused, split, window):
    n, log2 = 50_000, 5
    rng = np.random.default_rng(8)
    types = rng.choice([OP_CONTAINS, OP_INSERT, OP_REMOVE], size=n, p=[0.5, 0.4, 0.1])
    types = types.astype(np.uint8)
    keys = rng.integers(0, 3000, size=n).astype(np.uint32)
    keys[rng.random(n) < 0.2] = np.uint32(0xFFFFFFFF)
    o = OracleSet(log2)
    want = o.mixed(types, keys)
    s = Set(log2, max_window=window)
    s.set_tuning(fused_split=split)
    out = _bools(n, cuda)
    (s.execute_fused if fused else s.execute)(dev(types), dev(keys), out)
    cuda.cuda.synchronize()
    got = host(out, np.uint8)
    bad = np.nonzero(got != want)[0]
    assert len(bad) == 0, f"{len(bad)} mismatches, first {bad[:5]}"
    assert np.array_equal(s.dump(), o.dump())
    assert s.status() == 0


def test_set_batches_per_type_vs_oracle(cuda):
    """40/50/10 insert/contains/remove batches issued per op type (insert,
    contains, remove launches), uniform u32 keys, prefilled at load factor 1."""
    seed, log2 = 4, 8
    pre = W.set_prefill_keys(seed, 28 * (1 << log2))
    o = OracleSet(log2)
    s = Set(log2, pool_slabs=1 << 12)
    o.insert(pre)
    s.insert(dev(pre))
    for b in range(4):
        bt = W.set_mixed_batch(seed, b, 1 << 13)
        want = o.mixed(bt.types, bt.keys)
        got = np.empty(len(bt.keys), np.uint8)
        for t, call in ((OP_CONTAINS, s.contains), (OP_INSERT, s.insert), (OP_REMOVE, s.remove)):
            sel = np.nonzero(bt.types == t)[0]
            if len(sel) == 0:
                continue
            out = _bools(len(sel), cuda)
            call(dev(bt.keys[sel]), out)
            cuda.cuda.synchronize()
            got[sel] = host(out, np.uint8)
        assert np.array_equal(got, want)
    assert np.array_equal(s.dump(), o.dump())
    assert s.status() == 0


def test_pool_not_wasted_by_concurrent_inserts(cuda):
    """Two keys per head slot inserted in large batches: chains need about one
    overflow slab per bucket, and concurrent refills of a per-SM slab range
    must not abandon half-used chunks (the pool then runs out)."""
    import torch
    from lslab_b200 import Set
    log2 = 14
    buckets = 1 << log2
    nk = 2 * buckets * 28
    pool = int(1.55 * buckets) + 148 * 32
    s = Set(log2, pool)
    keys = np.unique(W.splitmix64(91, 0, 2 * nk).astype(np.uint32))[:nk]
    for off in range(0, nk, 1 << 18):
        s.insert(torch.from_numpy(keys[off:off + (1 << 18)].view(np.int32)).cuda())
    torch.cuda.synchronize()
    used, cap = s.pool_usage()
    assert s.status() == 0
    assert s.size() == len(keys)
    # Poisson(56) keys per bucket need ~1.47 overflow slabs per bucket; each
    # SM may hold one partly used chunk (at most 32 slabs) on top
    assert used <= int(1.55 * buckets) + 148 * 32, (used, buckets)


def test_set_warp_cooperative_probe_exact(cuda):
    keys = W.perm32(np.arange(50_000))
    s = Set(6, 1 << 12)
    s.insert(dev(keys))
    s.remove(dev(keys[::3]))
    o = OracleSet(6)
    o.insert(keys)
    o.remove(keys[::3])
    q = W.perm32(np.arange(0, 100_000, 2))
    want = o.contains(q)
    for wp in (1, 0):
        s.set_tuning(warp_probe=wp)
        out = cuda.zeros(len(q), dtype=cuda.uint8, device="cuda")
        s.contains(dev(q), out)
        cuda.cuda.synchronize()
        assert np.array_equal(host(out, np.uint8), want), f"warp_probe={wp}"
    assert s.status() == 0
