"""Maps with 32-bit values (lslab::map<K, unsigned>, the shape of the
reference's own benchmark): lsb_map_put_v32 / put_pairs_v32 / get_v32 /
update_v32 give the oracle's results narrowed to 32 bits, in the layouts of
cuda::std::pair<bool, uint32_t> and cuda::std::pair<uint64_t, uint32_t>."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from lslab_b200 import Map, _lib
from lslab_b200 import workload as W
from oracle import OracleMap

pytestmark = pytest.mark.gpu

R32 = np.dtype([("found", "u1"), ("pad", "u1", (3,)), ("value", "<u4")])
KV32 = np.dtype([("key", "<u8"), ("value", "<u4"), ("pad", "<u4")])


def _dev(a):
    import torch
    return torch.from_numpy(np.frombuffer(np.ascontiguousarray(a).tobytes(), np.uint8).copy()).cuda()


def _host(t, dtype):
    return t.cpu().numpy().view(dtype)


def _call(name, *args):
    rc = getattr(_lib.lib(), name)(*args)
    assert rc == _lib.LSB_OK, _lib.error_string(rc)


def test_v32_put_get_update_equal_the_oracle(cuda):
    log2, n = 10, 40_000
    rng = np.random.default_rng(32)
    keys = W.key_of_rank(32, rng.integers(0, 15_000, size=n).astype(np.uint64))
    vals = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
    m = Map(log2)
    o = OracleMap(log2)
    # SoA put (repeated keys: old values chain in index order)
    old = cuda.zeros(n * 4, dtype=cuda.uint8, device="cuda")
    # device copies held in variables until the calls are done (a temporary's
    # memory could be reused by the next allocation before the kernel runs)
    dk, dv = _dev(keys), _dev(vals)
    _call("lsb_map_put_v32", m.handle, dk.data_ptr(), dv.data_ptr(), old.data_ptr(), n, None)
    want_old = o.put(keys, vals.astype(np.uint64))
    cuda.cuda.synchronize()
    assert np.array_equal(_host(old, np.uint32), want_old.astype(np.uint32))
    # AoS put of pairs
    pk = W.key_of_rank(33, rng.integers(0, 15_000, size=n).astype(np.uint64))
    pv = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
    pairs = np.zeros(n, KV32)
    pairs["key"], pairs["value"] = pk, pv
    old2 = cuda.zeros(n * 4, dtype=cuda.uint8, device="cuda")
    dp = _dev(pairs)
    _call("lsb_map_put_pairs_v32", m.handle, dp.data_ptr(), old2.data_ptr(), n, None)
    want_old2 = o.put(pk, pv.astype(np.uint64))
    cuda.cuda.synchronize()
    assert np.array_equal(_host(old2, np.uint32), want_old2.astype(np.uint32))
    # update of pairs, half absent
    uk = np.concatenate([pk[:5000], W.absent_keys(34, 5000, np.concatenate([keys, pk]))])
    uv = rng.integers(0, 2**32, size=len(uk), dtype=np.uint64).astype(np.uint32)
    up = np.zeros(len(uk), KV32)
    up["key"], up["value"] = uk, uv
    uout = cuda.zeros(len(uk) * 8, dtype=cuda.uint8, device="cuda")
    du = _dev(up)
    _call("lsb_map_update_v32", m.handle, du.data_ptr(), uout.data_ptr(), len(uk), None)
    want_u = o.update(uk, uv.astype(np.uint64))
    cuda.cuda.synchronize()
    gu = _host(uout, R32)
    assert np.array_equal(gu["found"], want_u["found"])
    assert np.array_equal(gu["value"], want_u["value"].astype(np.uint32))
    # get, present and absent
    q = np.concatenate([keys[:10000], uk])
    gout = cuda.zeros(len(q) * 8, dtype=cuda.uint8, device="cuda")
    dq = _dev(q)
    _call("lsb_map_get_v32", m.handle, dq.data_ptr(), gout.data_ptr(), len(q), None)
    want_g = o.get(q)
    cuda.cuda.synchronize()
    g = _host(gout, R32)
    assert np.array_equal(g["found"], want_g["found"])
    assert np.array_equal(g["value"], want_g["value"].astype(np.uint32))
    assert (g["pad"] == 0).all()
    # the 64-bit calls read the same table
    k, v = m.dump()
    ok, ov = o.dump()
    assert np.array_equal(k, ok) and np.array_equal(v, ov)
    assert m.status() == 0
