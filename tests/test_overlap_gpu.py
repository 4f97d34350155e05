"""The two-stream window form (tuning overlap=1): each window's reads run in
the lean read kernel on the caller's stream while its mutations are listed,
probed, grouped and ordered on a second stream; the resolve step joins both.
Results must equal the oracle's op-index-order replay exactly, for mixed
conflict-heavy batches (reads after same-key mutations are rewritten by the
resolve step), hot keys whose groups take the multi-step ordering, type-sorted
read-mostly batches, sets, CUDA-graph replays (device-side window epochs,
through their wrap-around), and tables that alternate with the persistent
kernel."""
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


def _mixed(seed, n, key_space, mix=(0.5, 0.35, 0.15)):
    u = W.uniform01(seed, 0, n)
    types = np.searchsorted(np.cumsum(mix)[:-1], u, side="right").astype(np.uint8)
    keys = W.key_of_rank(seed, W.splitmix64(seed + 1, 0, n) % np.uint64(key_space))
    vals = W.splitmix64(seed + 2, 0, n)
    return types, keys, vals


def _check_map(m, o, got, want):
    assert same_results(got, want), first_mismatch(got, want)
    k, v = m.dump()
    ok, ov = o.dump()
    assert np.array_equal(k, ok) and np.array_equal(v, ov)
    assert m.status() == 0


@pytest.mark.parametrize("fused", [False, True])
@pytest.mark.parametrize("window", [0, 4096])
def test_overlap_mixed_conflicts(cuda, fused, window):
    n, log2 = 60_000, 6
    types, keys, vals = _mixed(5, n, key_space=300)
    o = OracleMap(log2)
    want = o.mixed(types, keys, vals)
    m = Map(log2, max_window=window)
    m.set_tuning(overlap=1)
    out = results_buf(n)
    dt, dk, dv = dev(types), dev(keys), dev(vals)
    (m.execute_fused if fused else m.execute)(dt, dk, dv, out)
    _sync()
    _check_map(m, o, results(out), want)


def test_overlap_hot_keys(cuda):
    """~100k mutations of one key in one window (the grid-barrier ordering
    steps of k_sort run while the read kernel holds SMs) plus 50 warm keys."""
    n = 200_000
    rng = np.random.default_rng(3)
    types = rng.choice([OP_GET, OP_PUT, OP_REMOVE], size=n, p=[0.6, 0.3, 0.1]).astype(np.uint8)
    keys = W.key_of_rank(9, rng.integers(0, 50, size=n))
    keys[rng.random(n) < 0.5] = np.uint64(0xDEADBEEF)
    vals = rng.integers(0, 2**63, size=n, dtype=np.int64).astype(np.uint64)
    o = OracleMap(8)
    want = o.mixed(types, keys, vals)
    m = Map(8)
    m.set_tuning(overlap=1)
    out = results_buf(n)
    dt, dk, dv = dev(types), dev(keys), dev(vals)
    m.execute_fused(dt, dk, dv, out)
    _sync()
    _check_map(m, o, results(out), want)


def test_overlap_type_sorted_zipf(cuda):
    """The headline shape at reduced size: a prefilled table, one 95/5 Zipf
    batch with every get before every put."""
    seed, log2, pre, n = 7, 16, 1 << 20, 1 << 18
    pk = W.prefill_keys(seed, pre)
    pv = W.prefill_values(pk)
    b = W.map_zipf_batch(seed, 0, n, pre, 0.99, (0.95, 0.05))
    o = OracleMap(log2)
    o.put(pk, pv)
    want = o.mixed(b.types, b.keys, b.vals)
    m = Map(log2, 1 << 18)
    m.put(dev(pk), dev(pv))
    m.set_tuning(overlap=1)
    out = results_buf(n)
    dt, dk, dv = dev(b.types), dev(b.keys), dev(b.vals)
    m.execute_fused(dt, dk, dv, out)
    _sync()
    _check_map(m, o, results(out), want)


def test_overlap_set_mixed(cuda):
    n, log2 = 50_000, 6
    rng = np.random.default_rng(12)
    types = rng.choice([0, 1, 2], size=n, p=[0.5, 0.35, 0.15]).astype(np.uint8)
    keys = rng.integers(0, 2000, size=n).astype(np.uint32)
    o = OracleSet(log2)
    want = o.mixed(types, keys)
    for fused in (False, True):
        s = Set(log2)
        s.set_tuning(overlap=1)
        out = cuda.zeros(n, dtype=cuda.uint8, device="cuda")
        dt, dk = dev(types), dev(keys)
        (s.execute_fused if fused else s.execute)(dt, dk, out)
        _sync()
        assert np.array_equal(host(out, np.uint8), want)
        assert np.array_equal(s.dump(), o.dump())
        assert s.status() == 0
        s.close()


def test_overlap_graph_replays_through_epoch_wrap(cuda):
    """A captured call of 1024 windows of 32 ops replayed 34 times on new
    inputs (34,816 windows: past the 32,767 device epochs, so the group tables
    are cleared once on the device), alternating with persistent-kernel calls:
    every result equals the oracle's replay of all batches in order."""
    import torch
    n, log2, wnd, reps = 32 * 1024, 6, 32, 34
    m = Map(log2, max_window=wnd)
    m.set_tuning(overlap=1)
    o = OracleMap(log2)
    d_t = torch.empty(n, dtype=torch.uint8, device="cuda")
    d_k = torch.empty(n, dtype=torch.int64, device="cuda")
    d_v = torch.empty(n, dtype=torch.int64, device="cuda")
    out = results_buf(n)
    g = m.capture_fused(d_t, d_k, d_v, out)
    for r in range(reps):
        types, keys, vals = _mixed(100 + r, n, key_space=500)
        d_t.copy_(dev(types))
        d_k.copy_(dev(keys))
        d_v.copy_(dev(vals))
        g.launch()
        _sync()
        want = o.mixed(types, keys, vals)
        got = results(out)
        assert same_results(got, want), f"replay {r}: " + first_mismatch(got, want)
        if r % 8 == 7:  # the persistent kernel on the same table and epoch counter
            types, keys, vals = _mixed(900 + r, 4096, key_space=500)
            m.set_tuning(overlap=0)
            out2 = results_buf(4096)
            dt, dk, dv = dev(types), dev(keys), dev(vals)
            m.execute_fused(dt, dk, dv, out2)
            _sync()
            m.set_tuning(overlap=1)
            want2 = o.mixed(types, keys, vals)
            got2 = results(out2)
            assert same_results(got2, want2), f"fused after {r}: " + first_mismatch(got2, want2)
    g.close()
    _check_map(m, o, results(out), want)


def test_overlap_trace_spans(cuda):
    """With tracing on, a two-stream call records each window's start, its
    read kernel, listing, probing, ordering and resolve ends (timing events,
    lsb_map_read_trace); the steps on each stream end in order, the resolve
    last, and the results stay exact."""
    n, log2 = 20_000, 8
    types, keys, vals = _mixed(11, n, key_space=500)
    o = OracleMap(log2)
    want = o.mixed(types, keys, vals)
    m = Map(log2, max_window=8192)
    m.set_tuning(overlap=1)
    m.set_trace(True)
    out = results_buf(n)
    m.execute_fused(dev(types), dev(keys), dev(vals), out)
    tr = m.read_trace()
    _sync()
    assert same_results(results(out), want), first_mismatch(results(out), want)
    nwin = -(-n // 8192)
    assert len(tr) == 6 * nwin
    for wi in range(nwin):
        pts = {(w, ph): ns for ns, w, ph in tr if (w & 31) == wi}
        start, reads, muts, done = pts[(wi, 0)], pts[(wi, 1)], pts[(wi, 2)], pts[(wi, 3)]
        listed, probed = pts[(wi | 32, 1)], pts[(wi | 32, 2)]
        assert start <= listed <= probed <= muts <= done
        assert start <= reads <= done
    m.set_trace(False)
    assert m.status() == 0
