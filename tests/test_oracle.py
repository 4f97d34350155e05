"""CPU tests of the oracle: pinned against golden vectors produced by the
reference's own kernels (tests/golden/make_golden.py), against the
reference's own known-answer tests, and against a dict replay."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import OracleMap, OracleSet, UmapReplay, ref_map_pool_bound
from lslab_b200 import workload as W

GOLD = Path(__file__).resolve().parent / "golden"


def _load(name):
    p = GOLD / name
    assert p.exists(), f"golden fixture {p} missing (tests/golden/make_golden.py)"
    return np.load(p)


def test_golden_map_gets():
    g = _load("map_gets.npz")
    m = OracleMap(int(g["log2"]))
    assert np.array_equal(m.put(g["put_keys"], g["put_vals"]), g["put_old"])
    r = m.get(g["get_keys"])
    assert np.array_equal(r["found"], g["get_found"])
    assert np.array_equal(r["value"], g["get_value"])
    k, v = m.dump()
    assert np.array_equal(k, g["dump_keys"]) and np.array_equal(v, g["dump_vals"])
    # the oracle allocates overflow slabs exactly as the reference's pool did
    assert m.slabs_used() == int(g["pool_used"])


def test_golden_map_put_remove():
    g = _load("map_put_remove.npz")
    m = OracleMap(int(g["log2"]))
    for i in range(int(g["steps"])):
        kind = str(g[f"s{i}_kind"])
        keys = g[f"s{i}_keys"]
        if kind == "put":
            assert np.array_equal(m.put(keys, g[f"s{i}_vals"]), g[f"s{i}_old"]), i
        else:
            r = (m.remove if kind == "remove" else m.get)(keys)
            assert np.array_equal(r["found"], g[f"s{i}_found"]), i
            assert np.array_equal(r["value"], g[f"s{i}_value"]), i
    k, v = m.dump()
    assert np.array_equal(k, g["dump_keys"]) and np.array_equal(v, g["dump_vals"])


def test_golden_map_warp_chain():
    g = _load("map_warp_chain.npz")
    m = OracleMap(4)
    assert np.array_equal(m.put(g["keys"], g["vals"]), g["old"])


def test_golden_set_batches():
    g = _load("set_batches.npz")
    s = OracleSet(int(g["log2"]))
    s.insert(g["pre"])
    for i in range(int(g["steps"])):
        kind = str(g[f"s{i}_kind"])
        out = getattr(s, kind)(g[f"s{i}_keys"])
        assert np.array_equal(out, g[f"s{i}_out"]), (i, kind)
    assert np.array_equal(s.dump(), g["dump"])


def test_golden_set_known_answer():
    g = _load("set_known_answer.npz")
    s = OracleSet(10)
    outs = []
    for rep in range(3):
        for name in ("insert", "contains", "remove", "contains"):
            outs.append(getattr(s, name)(g["keys"]))
    assert np.array_equal(np.stack(outs), g["outs"])


def test_reference_known_answer_tests():
    """test/set_test.cu:40-81 and test/slabunified_test.cu:42-89, full 100 reps."""
    s = OracleSet(10)
    keys = np.arange(1, 1025, dtype=np.uint32)
    for _ in range(100):
        assert s.insert(keys).all()
        assert s.contains(keys).all()
        assert s.remove(keys).all()
        assert not s.contains(keys).any()
    m = OracleMap(10)
    k = np.arange(1, 1025, dtype=np.uint64)
    for rep in range(100):
        old = m.put(k, np.full(1024, rep, np.uint64))
        if rep:
            assert (old == rep - 1).all()
        r = m.get(k)
        assert r["found"].all() and (r["value"] == rep).all()


def _dict_replay(types, keys, vals):
    d = {}
    found = np.zeros(len(keys), np.uint8)
    value = np.zeros(len(keys), np.uint64)
    for i, (t, k) in enumerate(zip(types.tolist(), keys.tolist())):
        if k in d:
            found[i], value[i] = 1, d[k]
        if t == W.OP_PUT:
            d[k] = int(vals[i])
        elif t == W.OP_REMOVE:
            d.pop(k, None)
        elif t == W.OP_UPDATE and k in d:
            d[k] = int(vals[i])
    return found, value, d


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_equals_dict_replay(seed):
    """Mixed get/put/remove/update with heavy key reuse: the slab-list oracle
    gives the same results as a plain dict replayed in index order (an update
    changes a present key's value and leaves an absent key absent)."""
    n = 20_000
    rng = np.random.default_rng(seed)
    types = rng.choice([0, 1, 2, 3], size=n, p=[0.4, 0.3, 0.15, 0.15]).astype(np.uint8)
    keys = W.key_of_rank(seed, rng.integers(0, 500, size=n))
    keys[rng.random(n) < 0.05] = np.uint64(0)
    vals = W.splitmix64(seed, 0, n)
    o = OracleMap(3)
    r = o.mixed(types, keys, vals)
    f, v, d = _dict_replay(types, keys, vals)
    assert np.array_equal(r["found"], f)
    assert np.array_equal(r["value"], v)
    k, vv = o.dump()
    assert len(k) == len(d)
    assert all(d[int(a)] == int(b) for a, b in zip(k, vv))


@pytest.mark.parametrize("shards,threads", [(1, 1), (4, 1), (4, 4)])
def test_unordered_map_replay_equals_oracle(shards, threads):
    """The std::unordered_map host replay (the reported CPU baseline) gives the
    oracle's results on a prefilled map under a mixed Zipf batch with
    removes and re-puts, single-threaded and one thread per shard."""
    seed, log2 = 5, 8
    pk = W.prefill_keys(seed, 1 << 12)
    pv = W.prefill_values(pk)
    o = OracleMap(log2)
    o.put(pk, pv)
    u = UmapReplay(pk, pv, shards=shards)
    for b in range(3):
        bt = W.map_zipf_batch(seed, b, 1 << 14, 1 << 13, 0.99, (0.5, 0.25, 0.1, 0.15),
                              type_sort=False)
        want = o.mixed(bt.types, bt.keys, bt.vals)
        dt, got = u.replay(bt.types, bt.keys, bt.vals, threads=threads)
        assert dt >= 0
        assert np.array_equal(got["found"], want["found"])
        assert np.array_equal(got["value"], want["value"])
    assert u.size() == len(o.dump()[0])
    u.close()


def test_oracle_multithreaded_equals_single():
    seed, log2 = 9, 10
    pk = W.prefill_keys(seed, 1 << 15)
    a, b = OracleMap(log2), OracleMap(log2)
    a.put(pk, W.prefill_values(pk))
    b.put(pk, W.prefill_values(pk))
    bt = W.map_zipf_batch(seed, 0, 1 << 16, 1 << 15, 0.99, (0.8, 0.15, 0.05), type_sort=False)
    ra = a.mixed(bt.types, bt.keys, bt.vals)
    rb = b.mixed(bt.types, bt.keys, bt.vals, threads=4)
    assert np.array_equal(ra, rb)
    ka, va = a.dump()
    kb, vb = b.dump()
    assert np.array_equal(ka, kb) and np.array_equal(va, vb)


def test_set_oracle_multithreaded_equals_single():
    bt = W.set_mixed_batch(5, 0, 1 << 15, type_sort=False)
    a, b = OracleSet(6), OracleSet(6)
    assert np.array_equal(a.mixed(bt.types, bt.keys), b.mixed(bt.types, bt.keys, threads=3))
    assert np.array_equal(a.dump(), b.dump())


def test_pool_bound_covers_reference_allocation():
    """The slab bound handed to the reference's allocator (so it never traps)
    is at least what the restated allocator uses."""
    log2 = 4
    keys = W.prefill_keys(3, 5000)
    m = OracleMap(log2)
    m.put(keys, keys)
    assert ref_map_pool_bound(log2, keys) >= m.slabs_used()
