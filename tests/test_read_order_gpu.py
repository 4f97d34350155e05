"""Reads in table-region order (tuning read_order): the lean read kernel takes
a call's reads through a device-built order (count per region, offsets,
scatter) instead of op order.  Results must be exactly those of op order and
of the oracle, for get and contains calls (odd sizes, repeats, absent keys,
32-bit values), for the reads of two-stream windows of mixed batches, and on
a table larger than L2."""
from __future__ import annotations

import numpy as np
import pytest

from lslab_b200 import Map, Set
from lslab_b200 import workload as W
from oracle import OracleMap, OracleSet
from tests.util import dev, host, results, results_buf, same_results, first_mismatch

pytestmark = pytest.mark.gpu


def _sync():
    import torch
    torch.cuda.synchronize()


@pytest.mark.parametrize("log2", [4, 10, 16])
def test_ordered_gets_equal_the_oracle(cuda, log2):
    rng = np.random.default_rng(log2)
    pk = W.prefill_keys(3, 40_000)
    pv = W.prefill_values(pk)
    n = 70_001  # not a multiple of the 4096-op counting chunk
    q = np.where(rng.random(n) < 0.7, pk[rng.integers(0, 3000, n)],
                 W.absent_keys(3, n, pk))  # repeats and misses
    o = OracleMap(log2)
    o.put(pk, pv)
    want = o.get(q)
    m = Map(log2, 1 << 14)
    m.put(dev(pk), dev(pv))
    for order in (1, 0):
        m.set_tuning(read_order=order)
        out = results_buf(n)
        dq = dev(q)
        m.get(dq, out)
        _sync()
        got = results(out)
        assert same_results(got, want), f"read_order={order}: " + first_mismatch(got, want)
    assert m.status() == 0


def test_ordered_gets_32bit_values(cuda):
    import torch
    from lslab_b200 import _lib
    log2, n = 8, 20_000
    k = W.prefill_keys(8, 5000)
    v = (k & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    m = Map(log2, 1 << 12)
    dk = dev(k)
    dv = torch.from_numpy(v.view(np.int32).copy()).cuda()
    old = torch.zeros(len(k), dtype=torch.int32, device="cuda")
    lib = _lib.lib()
    assert lib.lsb_map_put_v32(m.handle, dk.data_ptr(), dv.data_ptr(), old.data_ptr(), len(k),
                               None) == _lib.LSB_OK
    m.set_tuning(read_order=1)
    q = k[np.random.default_rng(8).integers(0, len(k), n)]
    out = torch.zeros(n, dtype=torch.int64, device="cuda")
    dq = dev(q)
    assert lib.lsb_map_get_v32(m.handle, dq.data_ptr(), out.data_ptr(), n, None) == _lib.LSB_OK
    _sync()
    r = host(out, np.uint64)
    assert np.all((r & np.uint64(0xFF)) == 1)
    assert np.array_equal((r >> np.uint64(32)).astype(np.uint32),
                          (q & np.uint64(0xFFFFFFFF)).astype(np.uint32))
    assert m.status() == 0


def test_ordered_contains(cuda):
    log2, n = 10, 50_000
    rng = np.random.default_rng(21)
    keys = rng.integers(0, 2**32, size=20_000, dtype=np.uint64).astype(np.uint32)
    q = np.concatenate([keys[rng.integers(0, len(keys), n // 2)],
                        rng.integers(0, 2**32, size=n - n // 2, dtype=np.uint64).astype(np.uint32)])
    o = OracleSet(log2)
    o.insert(keys)
    want = o.contains(q)
    s = Set(log2)
    s.insert(dev(keys))
    s.set_tuning(read_order=1)
    out = cuda.zeros(n, dtype=cuda.uint8, device="cuda")
    dq = dev(q)
    s.contains(dq, out)
    _sync()
    assert np.array_equal(host(out, np.uint8), want.astype(np.uint8))
    assert s.status() == 0


@pytest.mark.parametrize("fused", [False, True])
def test_ordered_reads_of_two_stream_windows(cuda, fused):
    n, log2 = 90_000, 7
    u = W.uniform01(31, 0, n)
    types = np.searchsorted(np.cumsum([0.6, 0.25, 0.15])[:-1], u, side="right").astype(np.uint8)
    keys = W.key_of_rank(31, W.splitmix64(32, 0, n) % np.uint64(2000))
    vals = W.splitmix64(33, 0, n)
    o = OracleMap(log2)
    want = o.mixed(types, keys, vals)
    m = Map(log2, max_window=1 << 15)
    m.set_tuning(overlap=1, read_order=1)
    out = results_buf(n)
    dt, dk, dv = dev(types), dev(keys), dev(vals)
    (m.execute_fused if fused else m.execute)(dt, dk, dv, out)
    _sync()
    got = results(out)
    assert same_results(got, want), first_mismatch(got, want)
    k, v = m.dump()
    ok, ov = o.dump()
    assert np.array_equal(k, ok) and np.array_equal(v, ov)
    assert m.status() == 0


def test_ordered_gets_on_a_table_above_l2(cuda):
    """2^19 buckets (240 MB of head slabs), a 2^17-get Zipf call: region
    order and op order give the same results."""
    log2, pre, n = 19, 1 << 21, 1 << 17
    pk = W.prefill_keys(44, pre)
    pv = W.prefill_values(pk)
    m = Map(log2, 1 << 18)
    for off in range(0, pre, 1 << 20):
        m.put(dev(pk[off:off + (1 << 20)]), dev(pv[off:off + (1 << 20)]))
    b = W.map_zipf_batch(44, 0, n, pre, 0.99, (1.0,))
    dq = dev(b.keys)
    outs = []
    for order in (1, 0):
        m.set_tuning(read_order=order)
        out = results_buf(n)
        m.get(dq, out)
        _sync()
        outs.append(results(out))
    assert same_results(outs[0], outs[1]), first_mismatch(outs[0], outs[1])
    assert outs[0]["found"].all()
    assert m.status() == 0
