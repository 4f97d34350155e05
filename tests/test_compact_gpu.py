"""Slab reclamation on the GPU: removed slots are reused by later inserts,
and lsb_map_compact / lsb_set_compact pack every chain and return emptied
overflow slabs to the pool, which hands them out before fresh ones.  Results
and contents always equal the oracle's replay; a churn of puts and removes
at a steady live count runs inside a fixed pool without running out."""
from __future__ import annotations

import numpy as np
import pytest

from lslab_b200 import Map, Set, OP_GET, OP_PUT, OP_REMOVE
from lslab_b200 import workload as W
from oracle import OracleMap, OracleSet
from tests.util import dev, host, results, results_buf, same_results, first_mismatch

pytestmark = pytest.mark.gpu


def _sync():
    import torch
    torch.cuda.synchronize()


def _same_contents(m, o):
    k, v = m.dump()
    ok, ov = o.dump()
    assert np.array_equal(k, ok) and np.array_equal(v, ov), "contents differ from the oracle"


@pytest.mark.parametrize("lock_mode", ["writer", "free"])
def test_compact_returns_slabs_and_keeps_contents(cuda, lock_mode):
    log2 = 8
    keys = W.prefill_keys(3, 200_000)  # ~780 keys a bucket: chains of ~28 slabs
    m = Map(log2, 1 << 14, lock_mode=lock_mode)
    o = OracleMap(log2)
    m.put(dev(keys), dev(keys ^ np.uint64(3)))
    o.put(keys, keys ^ np.uint64(3))
    gone = keys[np.random.default_rng(3).random(len(keys)) < 0.8]
    m.remove(dev(gone))
    o.remove(gone)
    used0, _ = m.pool_usage()
    freed = m.compact()
    used1, _ = m.pool_usage()
    assert freed > 0 and used1 == used0 - freed
    _same_contents(m, o)
    # gets after compaction see every surviving entry where it moved
    out = results_buf(20_000)
    m.get(dev(keys[:20_000]), out)
    _sync()
    w = o.get(keys[:20_000])
    g = results(out)
    assert same_results(g, w), first_mismatch(g, w)
    # inserts take the returned slabs before fresh ones
    more = W.prefill_keys(4, 50_000)
    m.put(dev(more), dev(more))
    o.put(more, more)
    used2, _ = m.pool_usage()
    assert used2 <= used0, (used0, used1, used2)
    _same_contents(m, o)
    assert m.status() == 0


def test_churn_at_steady_live_count_in_a_fixed_pool(cuda):
    """Each batch puts 20k fresh keys, removes the 20k put two batches
    before, and reads recent keys; 40 batches would need ~4x the pool
    without reclamation.  With a compaction every 5 batches the pool holds,
    nothing runs out, and every result equals the replay."""
    log2, per, nb = 10, 20_000, 40
    pool = 3000  # slabs; the live set needs ~(60k - 28k head slots) / 28 ~ 1.2k
    m = Map(log2, pool, max_window=1 << 16)
    o = OracleMap(log2)
    rng = np.random.default_rng(7)
    peak = 0
    for b in range(nb):
        new = W.prefill_keys(100 + b, per)
        old = W.prefill_keys(100 + b - 2, per) if b >= 2 else np.zeros(0, np.uint64)
        look = W.prefill_keys(100 + max(0, b - 1), 5000)
        t = np.concatenate([np.full(per, OP_PUT, np.uint8), np.full(len(old), OP_REMOVE, np.uint8),
                            np.full(len(look), OP_GET, np.uint8)])
        k = np.concatenate([new, old, look])
        o_ = rng.permutation(len(k))
        t, k = t[o_], k[o_]
        v = W.splitmix64(200 + b, 0, len(k))
        want = o.mixed(t, k, v)
        out = results_buf(len(k))
        (m.execute_fused if b % 2 else m.execute)(dev(t), dev(k), dev(v), out)
        _sync()
        got = results(out)
        assert same_results(got, want), f"batch {b}: " + first_mismatch(got, want)
        assert m.status() == 0, f"batch {b}: device status raised"
        if b % 5 == 4:
            m.compact()
        peak = max(peak, m.pool_usage()[0])
    assert peak <= pool
    _same_contents(m, o)


def test_set_compact(cuda):
    keys = W.perm32(np.arange(300_000))
    s = Set(8, 1 << 14)
    o = OracleSet(8)
    s.insert(dev(keys))
    o.insert(keys)
    gone = keys[::3]
    s.remove(dev(gone))
    o.remove(gone)
    assert s.compact() > 0
    assert np.array_equal(s.dump(), o.dump())
    out = cuda.zeros(len(keys), dtype=cuda.uint8, device="cuda")
    s.contains(dev(keys), out)
    _sync()
    assert np.array_equal(host(out, np.uint8), o.contains(keys))
    assert s.status() == 0
