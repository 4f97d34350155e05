"""The per-warp device API (include/lsb_device.cuh), the counterpart of the
reference's device methods map::get/put/update and set::contains/insert/
remove (include/lslab/map.h:92-183, set.h:64-90), called from test kernels
(tests/device/device_api_kernels.cu, compiled here with nvcc) on tables
made through the C-ABI.  One warp walking a batch 32 ops at a time is
sequential: results equal the oracle's replay.  Many warps on disjoint keys
are too.  Many warps on the same hot keys are concurrent: every get returns
a value some put wrote, and the table stays consistent."""
from __future__ import annotations

import ctypes as C
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from lslab_b200 import Map, Set, OP_GET, OP_PUT, OP_REMOVE, OP_UPDATE
from lslab_b200 import workload as W
from oracle import OracleMap, OracleSet
from tests.util import dev, host, results, results_buf, same_results, first_mismatch

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    out = tmp_path_factory.mktemp("devapi") / "libdevapi.so"
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cmd = [nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", str(ROOT / "include"), "-I", str(ROOT / "lslab_b200" / "csrc"),
           "-Xcompiler", "-fPIC", "-shared", str(ROOT / "tests" / "device" / "device_api_kernels.cu"),
           "-o", str(out), "-L", str(ROOT / "lslab_b200"), "-llsb",
           "-Xlinker", f"-rpath,{ROOT / 'lslab_b200'}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    L = C.CDLL(str(out))
    P = C.c_void_p
    L.dev_map_ops.argtypes = [P, P, P, P, P, C.c_uint32, C.c_int, P]
    L.dev_set_ops.argtypes = [P, P, P, P, C.c_uint32, C.c_int, P]
    return L


def _sync():
    import torch
    torch.cuda.synchronize()


# A warp's group of 32 ops runs one method call at a time (get, put, update,
# remove, as the test kernel calls them), each call in lane order: the
# order in which the group's ops take effect when they are sorted this way.
_METHOD_RANK = {OP_GET: 0, OP_PUT: 1, OP_UPDATE: 2, OP_REMOVE: 3}


def _method_order(t, *arrays):
    """Stable-sort every group of 32 ops by method rank, so index order is
    the order the test kernel applies them in."""
    rank = np.vectorize(_METHOD_RANK.get)(t) if len(t) else t
    grp = np.arange(len(t)) // 32
    o = np.lexsort((np.arange(len(t)), rank, grp))
    return (t[o],) + tuple(a[o] for a in arrays)


def _map_batch(seed, n, key_space):
    rng = np.random.default_rng(seed)
    t = rng.choice([OP_GET, OP_PUT, OP_REMOVE, OP_UPDATE], size=n,
                   p=[0.4, 0.3, 0.15, 0.15]).astype(np.uint8)
    k = W.key_of_rank(seed, rng.integers(0, key_space, size=n).astype(np.uint64))
    k[rng.random(n) < 0.02] = np.uint64(0)  # key 0 is an ordinary key
    v = W.splitmix64(seed + 1, 0, n)
    return _method_order(t, k, v)


def _want_map(o, t, k, v):
    """The oracle's replay with the device API's result conventions (a put
    reports its old value only)."""
    w = o.mixed(t, k, v)
    w = w.copy()
    w["found"][t == OP_PUT] = 0
    return w


@pytest.mark.parametrize("lock_mode", ["writer", "rw"])
def test_one_warp_is_sequential(cuda, lib, lock_mode):
    t, k, v = _map_batch(3, 6000, 300)
    m = Map(6, lock_mode=lock_mode)
    out = results_buf(len(k))
    dt, dk, dv = dev(t), dev(k), dev(v)  # held until the kernel has run
    assert lib.dev_map_ops(m.handle, dt.data_ptr(), dk.data_ptr(), dv.data_ptr(),
                           out.data_ptr(), len(k), 1, None) == 0
    _sync()
    want = _want_map(OracleMap(6), t, k, v)
    got = results(out)
    assert same_results(got, want), first_mismatch(got, want)
    o = OracleMap(6)
    o.mixed(t, k, v)
    kk, vv = m.dump()
    ok, ov = o.dump()
    assert np.array_equal(kk, ok) and np.array_equal(vv, ov)
    assert m.status() == 0


def test_many_warps_on_disjoint_keys(cuda, lib):
    """Each warp's 32 ops use keys no other warp touches: all warps run at
    once and every result still equals the replay."""
    n = 1 << 16
    rng = np.random.default_rng(5)
    t = rng.choice([OP_GET, OP_PUT, OP_REMOVE, OP_UPDATE], size=n,
                   p=[0.4, 0.3, 0.15, 0.15]).astype(np.uint8)
    # key j of group g: 4 keys a group, so lanes repeat keys (lane order matters)
    k = W.key_of_rank(7, (np.arange(n) // 32 * 4 + rng.integers(0, 4, size=n)).astype(np.uint64))
    v = W.splitmix64(8, 0, n)
    t, k, v = _method_order(t, k, v)
    m = Map(10, 1 << 14)
    out = results_buf(n)
    dt, dk, dv = dev(t), dev(k), dev(v)
    assert lib.dev_map_ops(m.handle, dt.data_ptr(), dk.data_ptr(), dv.data_ptr(),
                           out.data_ptr(), n, 0, None) == 0
    _sync()
    want = _want_map(OracleMap(10), t, k, v)
    got = results(out)
    assert same_results(got, want), first_mismatch(got, want)
    assert m.status() == 0


def test_many_warps_on_hot_keys_stay_consistent(cuda, lib):
    """All warps put and get 16 hot keys at once: a get sees absent (before
    any put of its key) or a value some put of that key wrote; afterwards
    every key holds one of its written values, and the batch API reads the
    same table."""
    n = 1 << 16
    rng = np.random.default_rng(9)
    t = np.where(rng.random(n) < 0.5, OP_PUT, OP_GET).astype(np.uint8)
    hot = W.key_of_rank(9, np.arange(16, dtype=np.uint64))
    k = hot[rng.integers(0, 16, size=n)]
    v = np.arange(1, n + 1, dtype=np.uint64)  # each put writes a distinct value
    m = Map(4)
    out = results_buf(n)
    dt, dk, dv = dev(t), dev(k), dev(v)
    assert lib.dev_map_ops(m.handle, dt.data_ptr(), dk.data_ptr(), dv.data_ptr(),
                           out.data_ptr(), n, 0, None) == 0
    _sync()
    got = results(out)
    written = {int(key): set(v[(t == OP_PUT) & (k == key)].tolist()) for key in hot}
    gets = np.nonzero(t == OP_GET)[0]
    for i in gets[:5000]:
        if got["found"][i]:
            assert int(got["value"][i]) in written[int(k[i])]
    kk, vv = m.dump()
    assert len(kk) == 16
    for key, val in zip(kk.tolist(), vv.tolist()):
        assert val in written[key]
    # the batch API agrees with what the device API left
    g = results_buf(16)
    m.get(dev(hot), g)
    _sync()
    r = results(g)
    assert r["found"].all()
    assert m.status() == 0


def test_set_device_api_one_warp(cuda, lib):
    rng = np.random.default_rng(11)
    n = 6000
    t = rng.choice([0, 1, 2], size=n, p=[0.4, 0.4, 0.2]).astype(np.uint8)
    k = W.perm32(rng.integers(0, 500, size=n))
    # contains, insert, remove: the kernel's call order within a group of 32
    o = np.lexsort((np.arange(n), t, np.arange(n) // 32))
    t, k = t[o], k[o]
    s = Set(5)
    out = cuda.zeros(n, dtype=cuda.uint8, device="cuda")
    dt, dk = dev(t), dev(k)
    assert lib.dev_set_ops(s.handle, dt.data_ptr(), dk.data_ptr(), out.data_ptr(),
                           n, 1, None) == 0
    _sync()
    o = OracleSet(5)
    want = o.mixed(t, k)
    assert np.array_equal(host(out, np.uint8), want)
    assert np.array_equal(s.dump(), o.dump())
    assert s.status() == 0
