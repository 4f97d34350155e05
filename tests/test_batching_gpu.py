"""The batching form on the GPU: many uneven batches through one fused
launch, CUDA-graph replays of the fused launch, and the autotuner — every
result and the final contents bit-exact against the oracle's sequential
replay."""
from __future__ import annotations

import numpy as np
import pytest

import lslab_b200 as L
from lslab_b200 import workload as W
from oracle import OracleMap
from tests.util import dev, results, results_buf, same_results, first_mismatch

pytestmark = pytest.mark.gpu


def _uneven_batches(seed, count, items):
    sizes = W.lognormal_sizes(seed, count, 512, 1.5, 1, 1 << 14)
    parts = []
    for b, n in enumerate(sizes):
        bt = W.map_zipf_batch(seed, b, int(n), items, 0.99, (0.8, 0.15, 0.05))
        parts.append(bt)
    types = np.concatenate([p.types for p in parts])
    keys = np.concatenate([p.keys for p in parts])
    vals = np.concatenate([p.vals for p in parts])
    return parts, types, keys, vals


def test_uneven_batches_in_one_launch_equal_sequential(cuda):
    seed, log2, items = 41, 12, 1 << 15
    parts, types, keys, vals = _uneven_batches(seed, 300, items)
    pk = W.prefill_keys(seed, items // 2)
    o = OracleMap(log2)
    o.put(pk, pk)
    fused, plain = L.Map(log2, max_window=1 << 16), L.Map(log2)
    for m in (fused, plain):
        m.put(dev(pk), dev(pk))
    want = o.mixed(types, keys, vals)
    out = results_buf(len(keys))
    fused.execute_fused(dev(types), dev(keys), dev(vals), out)
    # plain: one call per op type per batch, as the reference's API issues them
    got_plain = []
    for bt in parts:
        g = int(np.sum(bt.types == 0))
        p = int(np.sum(bt.types == 1))
        og = results_buf(g)
        oo = cuda.zeros(p, dtype=cuda.int64, device="cuda")
        orr = results_buf(len(bt.keys) - g - p)
        if g:
            plain.get(dev(bt.keys[:g]), og)
        if p:
            plain.put(dev(bt.keys[g:g + p]), dev(bt.vals[g:g + p]), oo)
        if len(bt.keys) - g - p:
            plain.remove(dev(bt.keys[g + p:]), orr)
        got_plain.append((og, oo, orr, g, p))
    cuda.cuda.synchronize()
    gf = results(out)
    assert same_results(gf, want), first_mismatch(gf, want)
    at = 0
    for (og, oo, orr, g, p), bt in zip(got_plain, parts):
        w = want[at:at + len(bt.keys)]
        if g:
            assert same_results(results(og), w[:g])
        if p:
            assert np.array_equal(oo.cpu().numpy().view(np.uint64), w["value"][g:g + p])
        if len(bt.keys) - g - p:
            assert same_results(results(orr), w[g + p:])
        at += len(bt.keys)
    k1, v1 = fused.dump()
    k2, v2 = plain.dump()
    ko, vo = o.dump()
    assert np.array_equal(k1, ko) and np.array_equal(v1, vo)
    assert np.array_equal(k2, ko) and np.array_equal(v2, vo)


def test_graph_replays_advance_state(cuda):
    """A captured fused launch replayed on new batch contents: every replay's
    results equal the sequential replay (device-side window epochs)."""
    seed, log2, n = 43, 10, 20_000
    o = OracleMap(log2)
    m = L.Map(log2, max_window=4096)
    t_buf = cuda.zeros(n, dtype=cuda.uint8, device="cuda")
    k_buf = cuda.zeros(n, dtype=cuda.int64, device="cuda")
    v_buf = cuda.zeros(n, dtype=cuda.int64, device="cuda")
    out = results_buf(n)
    g = m.capture_fused(t_buf, k_buf, v_buf, out)
    rng = np.random.default_rng(seed)
    for rep in range(6):
        types = rng.choice([0, 1, 2], size=n, p=[0.5, 0.35, 0.15]).astype(np.uint8)
        keys = W.key_of_rank(seed, rng.integers(0, 3000, size=n))
        vals = W.splitmix64(seed + rep, 0, n)
        t_buf.copy_(dev(types))
        k_buf.copy_(dev(keys))
        v_buf.copy_(dev(vals))
        g.launch()
        cuda.cuda.synchronize()
        want = o.mixed(types, keys, vals)
        got = results(out)
        assert same_results(got, want), f"replay {rep}: " + first_mismatch(got, want)
    g.close()
    k, v = m.dump()
    ko, vo = o.dump()
    assert np.array_equal(k, ko) and np.array_equal(v, vo)
    assert m.status() == 0


def test_autotune_keeps_single_application_state(cuda):
    seed, log2, items = 47, 11, 1 << 14
    _, types, keys, vals = _uneven_batches(seed, 60, items)
    o = OracleMap(log2)
    o.mixed(types, keys, vals)
    m = L.Map(log2, max_window=1 << 15)
    out = results_buf(len(keys))
    best = m.autotune(dev(types), dev(keys), dev(vals), out)
    assert best["block_threads"] in (128, 256, 512, 1024)
    assert best["overlap"] in (0, 1)
    assert best["prefetch"] in (0, 1, 2)
    assert m.tuning() == best
    k, v = m.dump()
    ko, vo = o.dump()
    assert np.array_equal(k, ko) and np.array_equal(v, vo)
    again = L.Map(log2)  # same size: starts from the tuned shape
    assert again.tuning() == best
    assert m.status() == 0
