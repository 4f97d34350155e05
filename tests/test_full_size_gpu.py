"""Parity at the benchmark configurations' own sizes.

The other GPU parity tests run small tables; these run each benchmark
configuration at its full size once and compare every result and the final
sorted contents with the oracle (and, where the batch has no cross-warp
same-key conflict, with the reference's own kernels too):

  1. map, 2^16 buckets, 2^20 keys inserted, 2^20 gets (half present) in
     2^16-op calls: this library == the reference's kernels == the oracle;
  2. map, 2^22 buckets prefilled with 2^26 keys, one 2^20-op 95/5 Zipf(0.99)
     batch, through the fused kernel and through the per-op-type calls;
  3. set, 2^18 buckets at 0.25 .. 4 keys per head-slab slot and 2^24 buckets
     (2.7 GB of head slabs) at 0.25, one 2^18-op 40/50/10 batch each;
  4. map, 2^24 buckets prefilled with the 2^26 most popular of 2^27 keys,
     256 uneven lognormal batches (80/15/5, Zipf 0.99) drained by one
     CUDA-graph-captured fused launch.

The oracle runs multi-threaded (buckets sharded over host threads, results
identical to the single-threaded replay)."""
from __future__ import annotations

import os

import numpy as np
import pytest

import oracle
from oracle import OracleMap, OracleSet, RefMap, ref_map_pool_bound
from lslab_b200 import Map, Set
from lslab_b200 import workload as W
from tests.util import dev, host, results, results_buf, same_results, first_mismatch

pytestmark = pytest.mark.gpu

THREADS = max(1, min(32, os.cpu_count() or 1))


def _sync():
    import torch
    torch.cuda.synchronize()


def _oracle_prefill(o, keys, vals):
    o.mixed(np.ones(len(keys), np.uint8), keys, vals, threads=THREADS)


def _map_prefill(m, keys, vals, chunk=1 << 24):
    for off in range(0, len(keys), chunk):
        m.put(dev(keys[off:off + chunk]), dev(vals[off:off + chunk]))
    _sync()
    assert m.status() == 0


def _same_contents(m, o):
    k, v = m.dump()
    ok, ov = o.dump()
    assert len(k) == len(ok), (len(k), len(ok))
    assert np.array_equal(k, ok), "final keys differ from the oracle"
    assert np.array_equal(v, ov), "final values differ from the oracle"


def test_cfg1_plain_gets_full_size_three_way(cuda):
    """2^16 buckets, 2^20 inserted keys (value = key ^ 0x9E3779B97F4A7C15),
    2^20 gets half present / half absent, one 2^16-op get call at a time:
    the reference's kernels, the oracle and this library agree on every
    result and on the final contents."""
    assert oracle.ref_available(), "oracle/_ref/liblslab_ref.so is missing (make -C oracle ref)"
    seed, log2, nk, bn = 1, 16, 1 << 20, 1 << 16
    pk = W.prefill_keys(seed, nk)
    pv = W.prefill_values(pk)
    ak = W.absent_keys(seed, nk // 2 + 4096, pk)[: nk // 2]
    rng = np.random.default_rng(seed)
    q = np.concatenate([pk[rng.permutation(nk)[: nk // 2]], ak])
    q = q[rng.permutation(len(q))]
    m = Map(log2)
    _map_prefill(m, pk, pv)
    ref = RefMap(log2, ref_map_pool_bound(log2, pk))
    ref_old = cuda.empty(nk, dtype=cuda.int64, device="cuda")
    ref.put(dev(pk), dev(pv), ref_old)
    o = OracleMap(log2)
    o.put(pk, pv)
    want = o.get(q)
    got_l = results_buf(len(q))
    got_r = results_buf(len(q))
    for off in range(0, len(q), bn):
        kq = dev(q[off:off + bn])
        m.get(kq, got_l[off:off + bn])
        ref.get(kq, got_r[off:off + bn])
    _sync()
    gl, gr = results(got_l), results(got_r)
    assert same_results(gl, want), first_mismatch(gl, want)
    assert np.array_equal(gr["found"], want["found"]), "reference found bits differ"
    hit = want["found"] == 1
    assert np.array_equal(gr["value"][hit], want["value"][hit]), "reference values differ"
    assert abs(hit.mean() - 0.5) < 1e-9
    _same_contents(m, o)
    rk, rv = ref.dump()
    k, v = m.dump()
    assert np.array_equal(rk, k) and np.array_equal(rv, v)
    assert m.status() == 0
    ref.close()


def test_cfg2_headline_batch_full_size(cuda):
    """2^22 buckets, 2^26-key prefill, one 2^20-op 95/5 Zipf(0.99) batch
    (gets then puts): the fused kernel and the per-op-type calls both equal
    the oracle on every result and on the final 2^26-entry contents."""
    seed, log2, pre, n = 7, 22, 1 << 26, 1 << 20
    pk = W.prefill_keys(seed, pre)
    pv = W.prefill_values(pk)
    b = W.map_zipf_batch(seed, 0, n, pre, 0.99, (0.95, 0.05))
    o = OracleMap(log2, 1 << 16)
    _oracle_prefill(o, pk, pv)
    want = o.mixed(b.types, b.keys, b.vals, threads=THREADS)
    g = int(np.sum(b.types == 0))
    for form in ("fused", "plain"):
        m = Map(log2, 1 << 20)
        _map_prefill(m, pk, pv)
        out = results_buf(n)
        if form == "fused":
            m.execute_fused(dev(b.types), dev(b.keys), dev(b.vals), out)
        else:
            m.get(dev(b.keys[:g]), out[:g])
            old = cuda.zeros(n - g, dtype=cuda.int64, device="cuda")
            m.put(dev(b.keys[g:]), dev(b.vals[g:]), old)
        _sync()
        got = results(out)
        if form == "plain":
            got = got.copy()
            ov = host(old, np.uint64)
            assert np.array_equal(ov, want["value"][g:]), "put old values differ"
            got["value"][g:] = ov
            got["found"][g:] = want["found"][g:]  # a put call returns the old value only
        assert same_results(got, want), f"{form}: " + first_mismatch(got, want)
        assert m.status() == 0
        _same_contents(m, o)
        m.close()


@pytest.mark.parametrize("log2,lf", [(18, 0.25), (18, 0.5), (18, 1.0), (18, 2.0), (18, 4.0),
                                     (24, 0.25)])
def test_cfg3_sets_full_size(cuda, log2, lf):
    """set<u32> prefilled to `lf` keys per head-slab slot (28 slots a slab),
    then one 2^18-op batch, 40% insert / 50% contains / 10% remove over the
    prefill keys and as many absent ones, type-sorted: fused == oracle on
    every result and on the final contents.  (At 2^24 buckets, the 2.7 GB
    table, the higher load factors need up to 1.9 G distinct keys, more than
    the host oracle holds in a test; they run in the benchmark only.)"""
    nk = int(lf * (1 << log2) * 28)
    keys = W.perm32(np.arange(nk, dtype=np.uint64))
    pool = max(4096, int(nk / 28 * 1.5) + (1 << log2) // 4)
    s = Set(log2, pool)
    for off in range(0, nk, 1 << 24):
        s.insert(dev(keys[off:off + (1 << 24)]))
    _sync()
    assert s.status() == 0
    o = OracleSet(log2, nk // 31 + 4096)
    o.mixed(np.ones(nk, np.uint8), keys, threads=THREADS)
    rng = np.random.default_rng(log2 * 100 + int(lf * 8))
    n = 1 << 18
    u = rng.random(n)
    ty = np.where(u < 0.4, 1, np.where(u < 0.9, 0, 2)).astype(np.uint8)
    ty = np.sort(ty, kind="stable")  # contains, insert, remove
    bk = W.perm32(rng.integers(0, 2 * nk, size=n, dtype=np.uint64))
    want = o.mixed(ty, bk, threads=THREADS)
    out = cuda.zeros(n, dtype=cuda.uint8, device="cuda")
    s.execute_fused(dev(ty), dev(bk), out)
    _sync()
    got = host(out, np.uint8)
    bad = np.nonzero(got != want)[0]
    assert len(bad) == 0, f"{len(bad)} results differ; first at {bad[0]}"
    assert s.status() == 0
    assert np.array_equal(s.dump(), o.dump()), "final set contents differ from the oracle"
    s.close()


def test_cfg4_uneven_batches_graph_full_size(cuda):
    """2^24 buckets prefilled with the 2^26 most popular of 2^27 keys; 256
    mixed batches (lognormal sizes, median 512, sigma 1.5, clipped to
    [1, 2^18]; 80/15/5 get/put/remove; Zipf 0.99) placed back to back and
    drained by one CUDA-graph-captured fused launch: every result and the
    final contents equal the oracle's replay of the batches in order."""
    seed, log2, items, pre, nb = 11, 24, 1 << 27, 1 << 26, 256
    sizes = W.lognormal_sizes(seed, nb, 512, 1.5, 1, 1 << 18)
    parts = [W.map_zipf_batch(seed, i, int(k), items, 0.99, (0.8, 0.15, 0.05))
             for i, k in enumerate(sizes)]
    types = np.concatenate([p.types for p in parts])
    keys = np.concatenate([p.keys for p in parts])
    vals = np.concatenate([p.vals for p in parts])
    n = len(keys)
    pk = W.key_of_rank(seed, np.arange(pre))
    m = Map(log2, 1 << 22)
    _map_prefill(m, pk, pk)
    o = OracleMap(log2, 1 << 16)
    _oracle_prefill(o, pk, pk)
    want = o.mixed(types, keys, vals, threads=THREADS)
    d_t, d_k, d_v = dev(types), dev(keys), dev(vals)
    out = results_buf(n)
    g = m.capture_fused(d_t, d_k, d_v, out)
    g.launch()
    _sync()
    g.close()
    got = results(out)
    assert same_results(got, want), first_mismatch(got, want)
    assert m.status() == 0
    _same_contents(m, o)
