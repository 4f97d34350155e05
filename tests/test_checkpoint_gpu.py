"""Checkpoints through the C-ABI (lsb_map_save / lsb_map_load and the set
forms): a table saved and loaded again holds the same entries; a file the
host writer produced loads, and a library-written file reads back on the host
with the same records; a corrupt file is refused (LSB_ERR_IO) and creates
nothing."""
from __future__ import annotations

import numpy as np
import pytest

from lslab_b200 import Map, Set, LsbError, _lib
from lslab_b200 import checkpoint as CK
from lslab_b200 import workload as W
from oracle import OracleMap
from tests.util import dev, results, results_buf, same_results, first_mismatch

pytestmark = pytest.mark.gpu


def _sync():
    import torch
    torch.cuda.synchronize()


def test_map_save_load_round_trip(cuda, tmp_path):
    log2 = 12
    k = W.prefill_keys(5, 300_000)  # ~73 keys a bucket: chains of several slabs
    v = W.splitmix64(6, 0, len(k))
    m = Map(log2, 1 << 14, lock_mode="free")
    m.put(dev(k), dev(v))
    m.remove(dev(k[::5]))
    assert m.status() == 0
    path = tmp_path / "m.ck"
    m.save(path)
    host = CK.read(path)
    keep = np.ones(len(k), bool)
    keep[::5] = False
    o = np.argsort(k[keep])
    assert np.array_equal(host.keys, k[keep][o]) and np.array_equal(host.values, v[keep][o])
    assert host.log2_buckets == log2 and host.pool_slabs == 1 << 14 and host.lock_mode == 1
    m2 = Map.load(path)
    assert m2.buckets() == 1 << log2
    k1, v1 = m.dump()
    k2, v2 = m2.dump()
    assert np.array_equal(k1, k2) and np.array_equal(v1, v2)
    # the loaded table works: gets see the saved values
    out = results_buf(1000)
    m2.get(dev(k[:1000]), out)
    _sync()
    ref = OracleMap(log2)
    ref.put(k[keep], v[keep])
    w = ref.get(k[:1000])
    g = results(out)
    assert same_results(g, w), first_mismatch(g, w)
    assert m2.status() == 0


def test_map_load_into_other_shape_and_host_written_file(cuda, tmp_path):
    k = W.prefill_keys(7, 50_000)
    v = W.prefill_values(k)
    path = tmp_path / "h.ck"
    CK.write(path, CK.Checkpoint(0, 20, k, v, pool_slabs=4096))
    m = Map.load(path, pool_slabs=1 << 16, lock_mode="writer")
    kk, vv = m.dump()
    o = np.argsort(k)
    assert np.array_equal(kk, k[o]) and np.array_equal(vv, v[o])
    assert m.buckets() == 1 << 20 and m.pool_usage()[1] == 1 << 16


def test_set_save_load_round_trip(cuda, tmp_path):
    keys = W.perm32(np.arange(400_000))
    s = Set(10, 1 << 16)
    s.insert(dev(keys))
    s.remove(dev(keys[::7]))
    path = tmp_path / "s.ck"
    s.save(path)
    s2 = Set.load(path)
    assert np.array_equal(s.dump(), s2.dump())
    keep = np.ones(len(keys), bool)
    keep[::7] = False
    assert np.array_equal(CK.read(path).keys, np.sort(keys[keep]))
    assert s2.status() == 0


def test_empty_and_corrupt_checkpoints(cuda, tmp_path):
    m = Map(6)
    p = tmp_path / "e.ck"
    m.save(p)
    e = Map.load(p)
    assert e.size() == 0 and e.buckets() == 64
    k = W.prefill_keys(9, 1000)
    m.put(dev(k), dev(k))
    p2 = tmp_path / "c.ck"
    m.save(p2)
    b = bytearray(p2.read_bytes())
    b[56 + 16 * 10] ^= 1
    p2.write_bytes(bytes(b))
    with pytest.raises(LsbError) as ei:
        Map.load(p2)
    assert ei.value.code == _lib.LSB_ERR_IO
    with pytest.raises(LsbError) as ei:
        Set.load(p)  # a map checkpoint is not a set checkpoint
    assert ei.value.code == _lib.LSB_ERR_IO
    with pytest.raises(LsbError):
        Map.load(tmp_path / "missing.ck")
