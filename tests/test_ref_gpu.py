"""Three-way parity on the GPU: the reference's own kernels (lslab built for
sm_100a, oracle/_ref), the oracle, and this library, on the same seeded
inputs.  Batches here are free of cross-warp same-key conflicts, where the
reference's result is unique; every get result and the final sorted
contents must be identical."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from oracle import OracleMap, OracleSet, RefMap, RefSet, ref_map_pool_bound
from lslab_b200 import Map, Set
from lslab_b200 import workload as W
from tests.util import dev, host, results, results_buf, same_results, first_mismatch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref(cuda):
    assert oracle.ref_available(), "oracle/_ref/liblslab_ref.so is missing (make -C oracle ref)"
    return True


def test_ref_known_answers(cuda, ref):
    """The reference's own tests, run on its kernels through the harness."""
    s = RefSet(10, 64)
    keys = dev(np.arange(1, 1025, dtype=np.uint32))
    r = cuda.zeros(1024, dtype=cuda.uint8, device="cuda")
    for rep in range(5):
        s.insert(keys, r)
        s.contains(keys, r)
        cuda.cuda.synchronize()
        assert (host(r, np.uint8) == 1).all()
        s.remove(keys, r)
        s.contains(keys, r)
        cuda.cuda.synchronize()
        assert (host(r, np.uint8) == 0).all()
    m = RefMap(10, 64)
    k = dev(np.arange(1, 1025, dtype=np.uint64))
    old = cuda.zeros(1024, dtype=cuda.int64, device="cuda")
    out = results_buf(1024)
    for rep in range(5):
        m.put(k, dev(np.full(1024, rep, np.uint64)), old)
        m.get(k, out)
        cuda.cuda.synchronize()
        if rep:
            assert (host(old, np.uint64) == rep - 1).all()
        g = results(out)
        assert g["found"].all() and (g["value"] == rep).all()


def test_map_plain_gets_three_way(cuda, ref):
    """Prefill distinct keys (value = key ^ 0x9E37...), then gets half present /
    half absent, in batches: reference == oracle == this library."""
    seed, log2, n = 101, 12, 1 << 16
    pk = W.prefill_keys(seed, n)
    pv = W.prefill_values(pk)
    ak = W.absent_keys(seed, n, pk)
    rm = RefMap(log2, ref_map_pool_bound(log2, pk))
    om = OracleMap(log2)
    lm = Map(log2)
    rold = cuda.zeros(n, dtype=cuda.int64, device="cuda")
    lold = cuda.zeros(n, dtype=cuda.int64, device="cuda")
    rm.put(dev(pk), dev(pv), rold)
    lm.put(dev(pk), dev(pv), lold)
    oold = om.put(pk, pv)
    cuda.cuda.synchronize()
    assert np.array_equal(host(rold, np.uint64), oold)
    assert np.array_equal(host(lold, np.uint64), oold)
    for b in range(4):
        q = np.concatenate([pk[b * 4096:(b + 1) * 4096], ak[b * 4096:(b + 1) * 4096]])
        q = q[np.argsort(W.splitmix64(seed + b, 0, len(q)))]
        want = om.get(q)
        ro, lo = results_buf(len(q)), results_buf(len(q))
        rm.get(dev(q), ro)
        lm.get(dev(q), lo)
        cuda.cuda.synchronize()
        rr, lr = results(ro), results(lo)
        # the reference leaves .second unwritten on a miss: compare it on hits only
        assert np.array_equal(rr["found"], want["found"])
        hit = want["found"] == 1
        assert np.array_equal(rr["value"][hit], want["value"][hit])
        assert same_results(lr, want), first_mismatch(lr, want)
    rk, rv = rm.dump()
    lk, lv = lm.dump()
    ok, ov = om.dump()
    assert np.array_equal(rk, ok) and np.array_equal(rv, ov)
    assert np.array_equal(lk, ok) and np.array_equal(lv, ov)


def test_map_put_update_remove_three_way(cuda, ref):
    """Conflict-free put batches (new keys and updates of existing ones), a
    remove batch through the REMOVE branch of the reference's traversal, then
    re-puts of removed keys (slot reuse): old values, remove results and final
    contents agree three ways."""
    seed, log2 = 202, 8
    base = W.prefill_keys(seed, 30_000)
    rm = RefMap(log2, ref_map_pool_bound(log2, np.concatenate([base, base])))
    om, lm = OracleMap(log2), Map(log2)
    batches = [base[:10_000], base[5_000:20_000], base[15_000:30_000]]
    for bi, keys in enumerate(batches):
        vals = W.splitmix64(seed + 10 + bi, 0, len(keys))
        ro = cuda.zeros(len(keys), dtype=cuda.int64, device="cuda")
        lo = cuda.zeros(len(keys), dtype=cuda.int64, device="cuda")
        rm.put(dev(keys), dev(vals), ro)
        lm.put(dev(keys), dev(vals), lo)
        want = om.put(keys, vals)
        cuda.cuda.synchronize()
        assert np.array_equal(host(ro, np.uint64), want)
        assert np.array_equal(host(lo, np.uint64), want)
    rk = base[::3]
    rr, lr = results_buf(len(rk)), results_buf(len(rk))
    rm.remove(dev(rk), rr)
    lm.remove(dev(rk), lr)
    want = om.remove(rk)
    cuda.cuda.synchronize()
    assert same_results(results(rr), want), first_mismatch(results(rr), want)
    assert same_results(results(lr), want), first_mismatch(results(lr), want)
    again = base[::6]
    vals = W.splitmix64(seed + 50, 0, len(again))
    ro = cuda.zeros(len(again), dtype=cuda.int64, device="cuda")
    lo = cuda.zeros(len(again), dtype=cuda.int64, device="cuda")
    rm.put(dev(again), dev(vals), ro)
    lm.put(dev(again), dev(vals), lo)
    want = om.put(again, vals)
    cuda.cuda.synchronize()
    assert np.array_equal(host(ro, np.uint64), want)
    assert np.array_equal(host(lo, np.uint64), want)
    k1, v1 = rm.dump()
    k2, v2 = lm.dump()
    k3, v3 = om.dump()
    assert np.array_equal(k1, k3) and np.array_equal(v1, v3)
    assert np.array_equal(k2, k3) and np.array_equal(v2, v3)


def test_map_in_warp_chain_matches_reference(cuda, ref):
    """32 puts of one key inside one warp: the reference serves them in lane
    order (include/lslab/detail/traverse.h:45-48), so put i returns value i-1;
    the oracle and this library give the same chain."""
    keys = np.full(32, 0x1234, np.uint64)
    vals = np.arange(100, 132, dtype=np.uint64)
    rm, om, lm = RefMap(4, 16), OracleMap(4), Map(4)
    ro = cuda.zeros(32, dtype=cuda.int64, device="cuda")
    lo = cuda.zeros(32, dtype=cuda.int64, device="cuda")
    rm.put(dev(keys), dev(vals), ro)
    lm.put(dev(keys), dev(vals), lo)
    want = om.put(keys, vals)
    cuda.cuda.synchronize()
    assert np.array_equal(host(ro, np.uint64), want)
    assert np.array_equal(host(lo, np.uint64), want)
    assert np.array_equal(want[1:], vals[:-1])


def test_set_three_way(cuda, ref):
    """Set batches issued per type (insert, contains, remove), distinct keys
    within each launch: reference == oracle == this library."""
    seed, log2 = 303, 9
    pre = W.set_prefill_keys(seed, 31 * (1 << log2))
    batches = [W.set_mixed_batch(seed, b, 1 << 12) for b in range(3)]
    inserts = np.concatenate([pre] + [bt.keys[bt.types == 1] for bt in batches])
    rs = RefSet(log2, ref_map_pool_bound(log2, inserts.astype(np.uint64)))
    os_, ls = OracleSet(log2), Set(log2)
    r = cuda.zeros(len(pre), dtype=cuda.uint8, device="cuda")
    l = cuda.zeros(len(pre), dtype=cuda.uint8, device="cuda")
    rs.insert(dev(pre), r)
    ls.insert(dev(pre), l)
    os_.insert(pre)
    for b, bt in enumerate(batches):
        for t, name in ((0, "contains"), (1, "insert"), (2, "remove")):
            k = np.unique(bt.keys[bt.types == t])
            k = k[np.argsort(W.splitmix64(seed + 7 * b + t, 0, len(k)))]
            want = getattr(os_, name)(k)
            rr = cuda.zeros(len(k), dtype=cuda.uint8, device="cuda")
            lr = cuda.zeros(len(k), dtype=cuda.uint8, device="cuda")
            getattr(rs, name)(dev(k), rr)
            getattr(ls, name)(dev(k), lr)
            cuda.cuda.synchronize()
            assert np.array_equal(host(rr, np.uint8), want), name
            assert np.array_equal(host(lr, np.uint8), want), name
    assert np.array_equal(rs.dump(), os_.dump())
    assert np.array_equal(ls.dump(), os_.dump())
