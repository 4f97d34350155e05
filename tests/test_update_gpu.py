"""GPU parity of map update (update-if-present, returning the old value):
the batched call (the reference's map::update<bs>, include/lslab/map.h:217-220,
with the semantics its device functor intends) and updates inside mixed
batches, whose effect depends on the last earlier put or remove of the same
key.  Every result and the final contents equal the oracle's replay."""
from __future__ import annotations

import numpy as np
import pytest

from lslab_b200 import Map, OP_GET, OP_PUT, OP_REMOVE, OP_UPDATE
from lslab_b200 import workload as W
from oracle import OracleMap
from tests.util import dev, results, results_buf, same_results, first_mismatch

pytestmark = pytest.mark.gpu


def _sync():
    import torch
    torch.cuda.synchronize()


def _pairs(keys, vals):
    return dev(np.stack([keys, vals], axis=1).reshape(-1))


def _same_contents(m, o):
    k, v = m.dump()
    ok, ov = o.dump()
    assert np.array_equal(k, ok) and np.array_equal(v, ov), "final contents differ"


def test_update_batch_present_and_absent(cuda):
    """Half the keys present: those get {1, old} and the new value, the rest
    {0, 0} and stay absent; repeated keys in one batch chain in index order."""
    rng = np.random.default_rng(3)
    log2 = 10
    present = W.prefill_keys(3, 20_000)
    absent = W.absent_keys(3, 20_000, present)
    m = Map(log2)
    o = OracleMap(log2)
    m.put(dev(present), dev(present ^ np.uint64(1)))
    o.put(present, present ^ np.uint64(1))
    keys = np.concatenate([present[rng.integers(0, len(present), 30_000)],
                           absent[rng.integers(0, len(absent), 30_000)]])
    keys = keys[rng.permutation(len(keys))]
    vals = W.splitmix64(4, 0, len(keys))
    out = results_buf(len(keys))
    m.update(_pairs(keys, vals), out)
    _sync()
    want = o.update(keys, vals)
    got = results(out)
    assert same_results(got, want), first_mismatch(got, want)
    assert want["found"].sum() > 0 and (want["found"] == 0).sum() > 0
    _same_contents(m, o)
    assert m.size() == len(present)
    assert m.status() == 0


def test_update_known_answer(cuda):
    """update of a present key returns its old value and changes it; of an
    absent key returns {0, 0} and inserts nothing; then get sees the result."""
    m = Map(4)
    m.put(dev(np.array([5], np.uint64)), dev(np.array([50], np.uint64)))
    out = results_buf(2)
    m.update(_pairs(np.array([5, 6], np.uint64), np.array([51, 61], np.uint64)), out)
    g = results_buf(2)
    m.get(dev(np.array([5, 6], np.uint64)), g)
    _sync()
    r = results(out)
    assert r["found"].tolist() == [1, 0] and r["value"].tolist() == [50, 0]
    gg = results(g)
    assert gg["found"].tolist() == [1, 0] and gg["value"].tolist() == [51, 0]


@pytest.mark.parametrize("window", [1 << 12, 1 << 16])
@pytest.mark.parametrize("fused", [True, False])
def test_updates_in_mixed_batches(cuda, window, fused):
    """Gets, puts, removes and updates interleaved over few keys (hot keys
    with thousands of members: every ordering path), split into windows."""
    rng = np.random.default_rng(5 + window)
    n, log2 = 120_000, 6
    t = rng.choice([OP_GET, OP_PUT, OP_REMOVE, OP_UPDATE], size=n,
                   p=[0.4, 0.2, 0.1, 0.3]).astype(np.uint8)
    k = W.key_of_rank(5, np.minimum(rng.zipf(1.3, size=n) - 1, 2000).astype(np.uint64))
    v = W.splitmix64(6, 0, n)
    pre = np.unique(k)[::3]
    o = OracleMap(log2)
    o.put(pre, pre)
    want = o.mixed(t, k, v)
    m = Map(log2, max_window=window)
    m.put(dev(pre), dev(pre))
    out = results_buf(n)
    (m.execute_fused if fused else m.execute)(dev(t), dev(k), dev(v), out)
    _sync()
    got = results(out)
    assert same_results(got, want), first_mismatch(got, want)
    _same_contents(m, o)
    assert m.status() == 0


def test_update_only_hot_key_runs(cuda):
    """One key carrying ~60% of a 2^18-op window, nearly all updates with
    rare puts and removes: its members span many runs of the multi-block
    ordering, and an update's presence comes from an earlier run."""
    rng = np.random.default_rng(9)
    n, log2 = 1 << 18, 8
    t = np.full(n, OP_UPDATE, np.uint8)
    t[rng.random(n) < 0.002] = OP_PUT
    t[rng.random(n) < 0.002] = OP_REMOVE
    t[rng.random(n) < 0.2] = OP_GET
    k = W.key_of_rank(9, rng.integers(0, 300, size=n).astype(np.uint64))
    k[rng.random(n) < 0.6] = np.uint64(1234)
    v = W.splitmix64(10, 0, n)
    want = OracleMap(log2).mixed(t, k, v)
    for fused in (True, False):
        m = Map(log2, max_window=1 << 18)
        out = results_buf(n)
        (m.execute_fused if fused else m.execute)(dev(t), dev(k), dev(v), out)
        _sync()
        got = results(out)
        assert same_results(got, want), f"fused={fused}: " + first_mismatch(got, want)
        assert m.status() == 0
