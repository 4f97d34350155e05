"""GPU parity of the map against the oracle (lslab's slab list restated on the
host, run in op-index order).  Integer results must be bit-exact."""
from __future__ import annotations

import numpy as np
import pytest

from lslab_b200 import Map, LsbError, STATUS_OOM, OP_GET, OP_PUT, OP_REMOVE
from lslab_b200 import workload as W
from oracle import OracleMap
from tests.util import dev, host, results, results_buf, same_results, first_mismatch

pytestmark = pytest.mark.gpu


def _sync():
    import torch
    torch.cuda.synchronize()


def test_get_put_known_answer(cuda):
    """test/slabunified_test.cu:42-89: put keys 1..1024 with value rep returns
    rep-1; get returns {true, rep}; 100 reps on 2^10 buckets."""
    m = Map(10)
    keys = dev(np.arange(1, 1025, dtype=np.uint64))
    old = cuda.zeros(1024, dtype=cuda.int64, device="cuda")
    out = results_buf(1024)
    for rep in range(100):
        vals = dev(np.full(1024, rep, np.uint64))
        m.put(keys, vals, old)
        m.get(keys, out)
        _sync()
        if rep:
            assert (host(old, np.uint64) == rep - 1).all()
        r = results(out)
        assert r["found"].all() and (r["value"] == rep).all()
    assert m.status() == 0


def test_small_plain_gets_vs_oracle(cuda):
    """Plain-method shape at small size: insert distinct splitmix64 keys with
    value = key ^ 0x9E3779B97F4A7C15, then gets half present, half absent."""
    seed, log2, n = 11, 10, 1 << 14
    pk = W.prefill_keys(seed, n)
    pv = W.prefill_values(pk)
    ak = W.absent_keys(seed, n, pk)
    q = np.concatenate([pk[: n // 2], ak[: n // 2]])
    q = q[np.argsort(W.splitmix64(seed + 99, 0, len(q)))]

    o = OracleMap(log2)
    o_old = o.put(pk, pv)
    want = o.get(q)

    m = Map(log2)
    old = cuda.zeros(n, dtype=cuda.int64, device="cuda")
    m.put(dev(pk), dev(pv), old)
    out = results_buf(len(q))
    m.get(dev(q), out)
    _sync()
    assert (host(old, np.uint64) == o_old).all()
    got = results(out)
    assert same_results(got, want), first_mismatch(got, want)
    k, v = m.dump()
    ok, ov = o.dump()
    assert np.array_equal(k, ok) and np.array_equal(v, ov)
    assert m.status() == 0


def _mixed_case(seed, n, key_space, mix=(0.5, 0.35, 0.15)):
    u = W.uniform01(seed, 0, n)
    cum = np.cumsum(mix)
    types = np.searchsorted(cum[:-1], u, side="right").astype(np.uint8)
    keys = W.key_of_rank(seed, (W.splitmix64(seed + 1, 0, n) % np.uint64(key_space)))
    vals = W.splitmix64(seed + 2, 0, n)
    return types, keys, vals


@pytest.mark.parametrize("fused,split,region", [(False, 100, 0), (True, 100, 0), (True, 0, 0),
                                                (True, 40, 0), (True, 0, 1), (True, 100, 1)])
@pytest.mark.parametrize("window", [0, 4096])
def test_mixed_conflicts_vs_oracle(cuda, fused, split, region, window):
    """Random get/put/remove order over a small key space (heavy same-key
    conflicts inside and across windows): every result and the final contents
    equal the sequential replay."""
    n, log2 = 60_000, 6
    types, keys, vals = _mixed_case(5, n, key_space=300)
    o = OracleMap(log2)
    want = o.mixed(types, keys, vals)
    m = Map(log2, max_window=window)
    m.set_tuning(fused_split=split, region_order=region)
    out = results_buf(n)
    run = m.execute_fused if fused else m.execute
    run(dev(types), dev(keys), dev(vals), out)
    _sync()
    got = results(out)
    assert same_results(got, want), first_mismatch(got, want)
    k, v = m.dump()
    ok, ov = o.dump()
    assert np.array_equal(k, ok) and np.array_equal(v, ov)
    assert m.status() == 0


@pytest.mark.parametrize("fused,block,split", [(False, 512, 100), (True, 128, 100),
                                               (True, 256, 100), (True, 512, 100),
                                               (True, 1024, 100), (True, 256, 0),
                                               (True, 1024, 0)])
def test_hot_key_big_groups(cuda, fused, block, split):
    """One key carries ~40k mutations in one window (the multi-step ordering
    of hot keys) and 50 keys ~800 each (block-wide ordering), interleaved
    with reads of them; every launch shape of the fused kernel."""
    n = 200_000
    rng = np.random.default_rng(3)
    types = rng.choice([OP_GET, OP_PUT, OP_REMOVE], size=n, p=[0.6, 0.3, 0.1]).astype(np.uint8)
    keys = W.key_of_rank(9, rng.integers(0, 50, size=n))
    keys[rng.random(n) < 0.5] = np.uint64(0xDEADBEEF)
    vals = rng.integers(0, 2**63, size=n, dtype=np.int64).astype(np.uint64)
    o = OracleMap(8)
    want = o.mixed(types, keys, vals)
    m = Map(8)
    m.set_tuning(block_threads=block, fused_split=split)
    out = results_buf(n)
    (m.execute_fused if fused else m.execute)(dev(types), dev(keys), dev(vals), out)
    _sync()
    got = results(out)
    assert same_results(got, want), first_mismatch(got, want)
    assert m.status() == 0


@pytest.mark.parametrize("fused,split,region", [(False, 100, 0), (True, 100, 0), (True, 0, 0),
                                                (True, 0, 1)])
def test_huge_skewed_groups(cuda, fused, split, region):
    """Groups far above the shared-memory sort size in one 2^20-op window:
    one key spread over the whole window, one packed densely into a narrow
    index range with a few strays far away (a very uneven spread of member
    indices), and a dozen Zipf-hot keys."""
    n = 1 << 20
    rng = np.random.default_rng(17)
    types = rng.choice([OP_GET, OP_PUT, OP_REMOVE], size=n, p=[0.5, 0.35, 0.15]).astype(np.uint8)
    keys = W.key_of_rank(4, rng.zipf(1.3, size=n).astype(np.uint64) % np.uint64(5000))
    keys[rng.random(n) < 0.2] = np.uint64(7)
    dense = slice(600_000, 640_000)
    keys[dense] = np.where(rng.random(40_000) < 0.8, np.uint64(8), keys[dense])
    keys[rng.integers(0, n, size=50)] = np.uint64(8)
    vals = rng.integers(0, 2**63, size=n, dtype=np.int64).astype(np.uint64)
    o = OracleMap(10)
    want = o.mixed(types, keys, vals)
    m = Map(10, max_window=n)
    m.set_tuning(fused_split=split, region_order=region)
    out = results_buf(n)
    (m.execute_fused if fused else m.execute)(dev(types), dev(keys), dev(vals), out)
    _sync()
    got = results(out)
    assert same_results(got, want), first_mismatch(got, want)
    k, v = m.dump()
    ok, ov = o.dump()
    assert np.array_equal(k, ok) and np.array_equal(v, ov)
    assert m.status() == 0


@pytest.mark.parametrize("split,region", [(0, 0), (100, 0), (0, 1)])
def test_type_sorted_batches_plain_equals_fused(cuda, split, region):
    """The 95/5 Zipf workload shape at small size: per-op-type calls (gets then
    puts) and the fused path give identical results, equal to the oracle."""
    seed, log2, items = 21, 12, 1 << 16
    pk = W.prefill_keys(seed, items)
    pv = W.prefill_values(pk)
    o = OracleMap(log2)
    o.put(pk, pv)
    a, b = Map(log2), Map(log2)
    b.set_tuning(fused_split=split, region_order=region)
    a.put(dev(pk), dev(pv))
    b.put(dev(pk), dev(pv))
    for bi in range(3):
        bt = W.map_zipf_batch(seed, bi, 1 << 15, items, 0.99, (0.95, 0.05))
        want = o.mixed(bt.types, bt.keys, bt.vals)
        ng = int(np.sum(bt.types == OP_GET))
        # plain: get launch then put launch
        outg = results_buf(ng)
        old = cuda.zeros(len(bt.keys) - ng, dtype=cuda.int64, device="cuda")
        a.get(dev(bt.keys[:ng]), outg)
        a.put(dev(bt.keys[ng:]), dev(bt.vals[ng:]), old)
        # fused
        outf = results_buf(len(bt.keys))
        b.execute_fused(dev(bt.types), dev(bt.keys), dev(bt.vals), outf)
        _sync()
        gf = results(outf)
        assert same_results(gf, want), first_mismatch(gf, want)
        gg = results(outg)
        assert same_results(gg, want[:ng]), first_mismatch(gg, want[:ng])
        assert np.array_equal(host(old, np.uint64), want["value"][ng:])
    ka, va = a.dump()
    kb, vb = b.dump()
    ko, vo = o.dump()
    assert np.array_equal(ka, ko) and np.array_equal(va, vo)
    assert np.array_equal(kb, ko) and np.array_equal(vb, vo)


@pytest.mark.parametrize("block,split", [(1024, 100), (512, 100), (512, 0)])
def test_queue_of_batches_in_one_launch(cuda, block, split):
    """The headline form: several type-sorted 95/5 batches back to back in one
    buffer, drained by one fused launch (one window per batch), give the
    results and contents of the per-op-type calls batch by batch and of the
    sequential replay."""
    seed, log2, items, nb, bn = 33, 12, 1 << 16, 6, 1 << 14
    pk = W.prefill_keys(seed, items)
    pv = W.prefill_values(pk)
    o = OracleMap(log2)
    o.put(pk, pv)
    q, p = Map(log2, max_window=bn), Map(log2)
    q.set_tuning(block_threads=block, fused_split=split)
    q.put(dev(pk), dev(pv))
    p.put(dev(pk), dev(pv))
    batches = [W.map_zipf_batch(seed, b, bn, items, 0.99, (0.95, 0.05)) for b in range(nb)]
    types = np.concatenate([b.types for b in batches])
    keys = np.concatenate([b.keys for b in batches])
    vals = np.concatenate([b.vals for b in batches])
    want = o.mixed(types, keys, vals)
    out = results_buf(len(keys))
    q.execute_fused(dev(types), dev(keys), dev(vals), out)
    _sync()
    got = results(out)
    assert same_results(got, want), first_mismatch(got, want)
    for bi, bt in enumerate(batches):
        ng = int(np.sum(bt.types == OP_GET))
        outg = results_buf(ng)
        old = cuda.zeros(bn - ng, dtype=cuda.int64, device="cuda")
        p.get(dev(bt.keys[:ng]), outg)
        p.put(dev(bt.keys[ng:]), dev(bt.vals[ng:]), old)
        _sync()
        w = want[bi * bn:(bi + 1) * bn]
        assert same_results(results(outg), w[:ng]), first_mismatch(results(outg), w[:ng])
        assert np.array_equal(host(old, np.uint64), w["value"][ng:])
    kq, vq = q.dump()
    kp, vp = p.dump()
    ko, vo = o.dump()
    assert np.array_equal(kq, ko) and np.array_equal(vq, vo)
    assert np.array_equal(kp, ko) and np.array_equal(vp, vo)
    assert q.status() == 0 and p.status() == 0


def test_remove_then_reinsert(cuda):
    """Remove half, re-put some (same-key revival), get all; also the
    AoS put form (map.h:189-192)."""
    n, log2 = 20_000, 8
    keys = W.prefill_keys(31, n)
    vals = W.prefill_values(keys)
    o = OracleMap(log2)
    m = Map(log2)
    pairs = np.stack([keys, vals], axis=1).reshape(-1)
    old = cuda.zeros(n, dtype=cuda.int64, device="cuda")
    m.put_pairs(dev(pairs), old)
    o.put(keys, vals)
    rk = keys[::2]
    out = results_buf(len(rk))
    m.remove(dev(rk), out)
    want = o.remove(rk)
    _sync()
    got = results(out)
    assert same_results(got, want), first_mismatch(got, want)
    again = keys[::4]
    nv = W.splitmix64(77, 0, len(again))
    old2 = cuda.zeros(len(again), dtype=cuda.int64, device="cuda")
    m.put(dev(again), dev(nv), old2)
    want_old = o.put(again, nv)
    q = np.concatenate([keys, W.absent_keys(31, 1000, keys)])
    outq = results_buf(len(q))
    m.get(dev(q), outq)
    wq = o.get(q)
    _sync()
    assert np.array_equal(host(old2, np.uint64), want_old)
    gq = results(outq)
    assert same_results(gq, wq), first_mismatch(gq, wq)
    k, v = m.dump()
    ok, ov = o.dump()
    assert np.array_equal(k, ok) and np.array_equal(v, ov)


def test_long_chains_and_edge_keys(cuda):
    """Tiny bucket array so chains grow many slabs deep; keys 0 and 2^64-1 are
    ordinary keys (no sentinel)."""
    log2 = 2
    keys = np.concatenate([np.array([0, 2**64 - 1], np.uint64), W.prefill_keys(41, 3000)])
    vals = np.concatenate([np.array([0, 2**64 - 1], np.uint64), W.splitmix64(42, 0, 3000)])
    o = OracleMap(log2)
    m = Map(log2, pool_slabs=1024)
    old = cuda.zeros(len(keys), dtype=cuda.int64, device="cuda")
    m.put(dev(keys), dev(vals), old)
    o.put(keys, vals)
    out = results_buf(len(keys))
    m.get(dev(keys), out)
    _sync()
    got = results(out)
    want = o.get(keys)
    assert same_results(got, want), first_mismatch(got, want)
    used, cap = m.pool_usage()
    assert used >= (len(keys) // 28) - 4 and cap == 1024
    assert m.status() == 0


def test_pool_exhaustion_reports_oom(cuda):
    """A pool too small for the inserts: the device raises OOM in the status
    word (the reference traps instead); nothing faults."""
    m = Map(1, pool_slabs=2)
    keys = W.prefill_keys(51, 2000)
    m.put(dev(keys), dev(keys))
    st = m.status()
    assert st & STATUS_OOM
    assert m.status() == 0  # cleared by the read


@pytest.mark.parametrize("mode", ["free", "rw"])
def test_lock_modes_agree(cuda, mode):
    n, log2 = 40_000, 5
    types, keys, vals = _mixed_case(61, n, key_space=2000)
    o = OracleMap(log2)
    want = o.mixed(types, keys, vals)
    m = Map(log2, lock_mode=mode)
    out = results_buf(n)
    m.execute(dev(types), dev(keys), dev(vals), out)
    _sync()
    got = results(out)
    assert same_results(got, want), first_mismatch(got, want)
    k, v = m.dump()
    ok, ov = o.dump()
    assert np.array_equal(k, ok) and np.array_equal(v, ov)
    assert m.status() == 0


def test_empty_and_bad_arguments(cuda):
    m = Map(4)
    e = cuda.empty(0, dtype=cuda.int64, device="cuda")
    m.get(e, results_buf(0), size=0)
    m.put(e, e, None, size=0)
    with pytest.raises(LsbError):
        m.get(0, 0, size=5)  # null keys
    with pytest.raises(LsbError):
        Map(0)  # zero log2 buckets
    assert m.buckets() == 16


@pytest.mark.parametrize("block", [128, 256, 1024])
@pytest.mark.parametrize("prefetch", [0, 1, 2])
@pytest.mark.parametrize("chunk", [0, 32, 2048])
@pytest.mark.parametrize("split", [0, 100])
@pytest.mark.parametrize("dedup", [0, 1])
def test_every_tuning_is_exact(cuda, block, prefetch, chunk, split, dedup):
    """Launch tuning never changes results (fused and per-phase paths),
    in-warp deduplication of same-key lookups included."""
    n, log2 = 40_000, 6
    types, keys, vals = _mixed_case(71, n, key_space=1500)
    want = OracleMap(log2).mixed(types, keys, vals)
    for fused in (True, False):
        m = Map(log2, max_window=8192)
        m.set_tuning(block_threads=block, prefetch=prefetch, chunk=chunk, fused_split=split,
                     dedup=dedup)
        out = results_buf(n)
        (m.execute_fused if fused else m.execute)(dev(types), dev(keys), dev(vals), out)
        _sync()
        got = results(out)
        assert same_results(got, want), f"fused={fused}: " + first_mismatch(got, want)
        assert m.status() == 0


@pytest.mark.parametrize("prefetch", [0, 2])
def test_dedup_on_hot_keys(cuda, prefetch):
    """In-warp deduplication (lanes with the same key share one lookup) on a
    batch where most warps carry repeated keys: a Zipf(1.2) mix over 64 keys
    with gets, puts and removes interleaved, several windows, reads-only
    calls too.  Results and final contents equal the oracle's replay, on the
    fused and the per-phase paths."""
    rng = np.random.default_rng(83)
    n, log2 = 200_000, 5
    ranks = np.minimum(rng.zipf(1.2, size=n) - 1, 63).astype(np.uint64)
    keys = W.key_of_rank(83, ranks)
    types = rng.choice([OP_GET, OP_PUT, OP_REMOVE], size=n, p=[0.7, 0.2, 0.1]).astype(np.uint8)
    vals = rng.integers(0, 2**63, size=n, dtype=np.int64).astype(np.uint64)
    o = OracleMap(log2)
    want = o.mixed(types, keys, vals)
    gets = W.key_of_rank(83, np.arange(80, dtype=np.uint64))
    want_gets = o.get(gets)
    for fused in (True, False):
        m = Map(log2, max_window=1 << 15)
        m.set_tuning(dedup=1, prefetch=prefetch)
        out = results_buf(n)
        (m.execute_fused if fused else m.execute)(dev(types), dev(keys), dev(vals), out)
        g_out = results_buf(len(gets))
        m.get(dev(gets), g_out)
        _sync()
        got = results(out)
        assert same_results(got, want), f"fused={fused}: " + first_mismatch(got, want)
        gg = results(g_out)
        assert same_results(gg, want_gets), first_mismatch(gg, want_gets)
        k, v = m.dump()
        ok, ov = o.dump()
        assert np.array_equal(k, ok) and np.array_equal(v, ov)
        assert m.status() == 0


def test_lock_free_inserts_do_not_waste_slabs(cuda):
    """LSB_LOCK_FREE map, 200k distinct keys into 256 buckets in one call:
    many inserts race to grow each chain; none is lost and the pool use stays
    near one slab per 28 keys (racing inserts keep and append their slabs)."""
    log2, n = 8, 200_000
    keys = W.prefill_keys(67, n)
    needed = n // 28 - (1 << log2)
    m = Map(log2, needed + 3000, lock_mode="free")
    m.put(dev(keys), dev(keys))
    assert m.status() == 0
    assert m.size() == n
    used, _ = m.pool_usage()
    assert used <= needed + 2 * (1 << log2) + 1500, (used, needed)
    o = OracleMap(log2)
    o.put(keys, keys)
    k, v = m.dump()
    ok, ov = o.dump()
    assert np.array_equal(k, ok) and np.array_equal(v, ov)


def test_warp_cooperative_probe_reads_exact(cuda):
    """The warp-cooperative slab probe (tuning warp_probe=1, the reference's
    probe structure) answers read-only batches exactly like the default
    probe: long chains, absent keys, keys repeated inside warps, key 0."""
    log2 = 6
    keys = W.prefill_keys(91, 40_000)  # ~625 keys a bucket: chains of ~23 slabs
    m = Map(log2, 1 << 13)
    m.put(dev(keys), dev(keys ^ np.uint64(5)))
    m.remove(dev(keys[::7]))
    o = OracleMap(log2)
    o.put(keys, keys ^ np.uint64(5))
    o.remove(keys[::7])
    rng = np.random.default_rng(91)
    q = np.concatenate([keys[rng.integers(0, len(keys), 30_000)], W.absent_keys(92, 5000, keys),
                        np.zeros(100, np.uint64), np.repeat(keys[:50], 20)])
    want = o.get(q)
    for wp in (1, 0):
        m.set_tuning(warp_probe=wp)
        out = results_buf(len(q))
        m.get(dev(q), out)
        _sync()
        got = results(out)
        assert same_results(got, want), f"warp_probe={wp}: " + first_mismatch(got, want)
    assert m.status() == 0
