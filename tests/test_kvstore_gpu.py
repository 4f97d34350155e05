"""KV store over the map (lsb_kvs_*): variable-size byte values in a device
heap.  Every get equals a Python dict replayed over the same puts and
removes; garbage accounting and heap compaction keep the contents."""
from __future__ import annotations

import numpy as np
import pytest

from lslab_b200 import KVStore, LsbError, _lib
from lslab_b200 import workload as W
from tests.util import dev, host

pytestmark = pytest.mark.gpu


def _sync():
    import torch
    torch.cuda.synchronize()


def _pack(values):
    off = np.zeros(len(values) + 1, np.uint64)
    off[1:] = np.cumsum([len(v) for v in values])
    buf = np.frombuffer(b"".join(values), np.uint8) if off[-1] else np.zeros(1, np.uint8)
    return buf, off


def _get_all(kv, keys, cuda):
    """Values as bytes (None when absent), through lsb_kvs_get."""
    n = len(keys)
    lens = cuda.zeros(n, dtype=cuda.int32, device="cuda")
    offs = cuda.zeros(n, dtype=cuda.int64, device="cuda")
    found = cuda.zeros(n, dtype=cuda.uint8, device="cuda")
    dk = dev(keys)
    total = kv.get(dk, lens, offs)
    dst = cuda.zeros(max(1, total), dtype=cuda.uint8, device="cuda")
    total2 = kv.get(dk, lens, offs, dst, total, found_out=found)
    assert total2 == total
    _sync()
    F = host(found, np.uint8)
    L = host(lens, np.uint32)
    O = host(offs, np.uint64)
    D = host(dst, np.uint8).tobytes()
    return [D[int(o):int(o) + int(l)] if f else None for f, o, l in zip(F, O, L)], L


def _values(rng, n, maxlen):
    lens = rng.integers(0, maxlen + 1, size=n)
    return [rng.integers(0, 256, size=int(l), dtype=np.uint8).tobytes() for l in lens]


def test_put_get_remove_equal_a_dict(cuda):
    rng = np.random.default_rng(1)
    kv = KVStore(10, 1 << 24)
    ref = {}
    keys_all = W.prefill_keys(1, 3000)
    for rnd in range(4):
        ks = keys_all[rng.integers(0, len(keys_all), size=2000)]
        vs = _values(rng, len(ks), 700)
        buf, off = _pack(vs)
        kv.put(dev(ks), dev(buf), dev(off))
        for k, v in zip(ks.tolist(), vs):
            ref[k] = v  # index order: the last put of a key wins
        gone = keys_all[rng.integers(0, len(keys_all), size=300)]
        found = cuda.zeros(len(gone), dtype=cuda.uint8, device="cuda")
        present_before = {k: (k in ref) for k in gone.tolist()}
        kv.remove(dev(gone), found)
        _sync()
        f = host(found, np.uint8)
        seen = set()
        for i, k in enumerate(gone.tolist()):
            want = present_before[k] and k not in seen
            assert bool(f[i]) == want
            seen.add(k)
            ref.pop(k, None)
        got, lens = _get_all(kv, keys_all, cuda)
        for k, g in zip(keys_all.tolist(), got):
            assert g == ref.get(k)
    assert kv.size() == len(ref)
    u = kv.usage()
    assert 0 < u["heap_dead"] <= u["heap_used"] <= u["heap_cap"]
    # compaction keeps every value and drops the garbage
    kv.compact()
    u2 = kv.usage()
    assert u2["heap_dead"] == 0 and u2["heap_used"] == sum(len(v) for v in ref.values())
    got, _ = _get_all(kv, keys_all, cuda)
    for k, g in zip(keys_all.tolist(), got):
        assert g == ref.get(k)


def test_heap_full_is_refused_without_effect(cuda):
    kv = KVStore(6, 4096)
    ks = W.prefill_keys(2, 3)
    buf, off = _pack([b"a" * 2000, b"b" * 2000, b"c" * 200])
    with pytest.raises(LsbError) as e:
        kv.put(dev(ks), dev(buf), dev(off))
    assert e.value.code == _lib.LSB_ERR_OOM
    assert kv.size() == 0 and kv.usage()["heap_used"] == 0
    buf, off = _pack([b"x" * 1000])
    kv.put(dev(ks[:1]), dev(buf), dev(off))
    got, _ = _get_all(kv, ks, cuda)
    assert got[0] == b"x" * 1000 and got[1] is None
