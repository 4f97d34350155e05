"""GPU tests of the serving loop (lsb_serve_*): a persistent kernel admitting
waves of queued requests.  Results must equal a sequential replay of the
requests in submission order (the oracle), each request's results must be
the same alone and in the mix, and admission must refuse what the slab pool
cannot hold without raising a device error."""
from __future__ import annotations

import time

import numpy as np
import pytest

from lslab_b200 import Map, Server, OP_GET, OP_PUT, OP_REMOVE
from lslab_b200 import _lib
from lslab_b200 import workload as W
from oracle import OracleMap
from tests.util import dev, same_results, first_mismatch

pytestmark = pytest.mark.gpu


def _requests(seed, count, max_n, key_space, mix=(0.5, 0.35, 0.15)):
    rng = np.random.default_rng(seed)
    reqs = []
    for _ in range(count):
        n = int(rng.integers(1, max_n + 1))
        t = rng.choice([OP_GET, OP_PUT, OP_REMOVE], size=n, p=list(mix)).astype(np.uint8)
        k = W.key_of_rank(seed, rng.integers(0, key_space, size=n).astype(np.uint64))
        v = rng.integers(0, 2**63, size=n, dtype=np.int64).astype(np.uint64)
        reqs.append((t, k, v))
    return reqs


def _submit_all(srv, reqs):
    tickets = []
    for t, k, v in reqs:
        for _ in range(100000):
            tk = srv.submit(t, k, v)
            if tk is not None:
                break
            time.sleep(0.0005)
        assert tk is not None, "queue stayed full"
        tickets.append(tk)
    return tickets


def _take_all(srv, reqs, tickets, timeout_s=60.0):
    out, status = [], []
    t_end = time.time() + timeout_s
    for (t, k, v), tk in zip(reqs, tickets):
        while not srv.done(tk):
            assert time.time() < t_end, "request did not finish"
            time.sleep(0.0002)
        r, st = srv.take(tk, len(k))
        out.append(r)
        status.append(st)
    return out, status


def test_serve_matches_sequential_replay(cuda):
    """Overlapping keys across requests: every result equals the replay of
    all requests one after another in submission order."""
    reqs = _requests(3, 300, 600, key_space=400)
    m = Map(8, max_window=1 << 16)
    srv = Server(m, max_wave_ops=1 << 14, ring_requests=1024, arena_ops=1 << 18)
    srv.start()
    tickets = _submit_all(srv, reqs)
    got, status = _take_all(srv, reqs, tickets)
    stats = srv.stop()
    srv.close()
    assert all(s == 0 for s in status)
    o = OracleMap(8)
    want = o.mixed(np.concatenate([r[0] for r in reqs]), np.concatenate([r[1] for r in reqs]),
                   np.concatenate([r[2] for r in reqs]))
    g = np.concatenate(got)
    assert same_results(g, want), first_mismatch(g, want)
    k, v = m.dump()
    ok, ov = o.dump()
    assert np.array_equal(k, ok) and np.array_equal(v, ov)
    assert stats["requests"] == len(reqs) and stats["state"] == 2
    assert m.status() == 0


def test_serve_alone_equals_mix(cuda):
    """Requests on disjoint keys: each request's results are the same when it
    runs alone (one request per wave) and mixed with the others (waves that
    hold many requests)."""
    base = _requests(5, 120, 800, key_space=50)
    reqs = [(t, k ^ np.uint64((i + 1) << 40), v) for i, (t, k, v) in enumerate(base)]
    runs = []
    for mode in ("alone", "mix"):
        m = Map(10, max_window=1 << 16)
        srv = Server(m, max_wave_ops=1 << 14, ring_requests=1024, arena_ops=1 << 18)
        srv.start()
        if mode == "alone":
            res = []
            for r in reqs:
                tk = _submit_all(srv, [r])
                g, st = _take_all(srv, [r], tk)
                assert st == [0]
                res += g
        else:
            tk = _submit_all(srv, reqs)
            res, st = _take_all(srv, reqs, tk)
            assert all(s == 0 for s in st)
        stats = srv.stop()
        srv.close()
        runs.append((res, stats))
        assert m.status() == 0
    (alone, sa), (mix, sm) = runs
    assert sa["waves"] == len(reqs)
    assert sm["waves"] < len(reqs), "the mixed run never put two requests in one wave"
    for i, (a, b) in enumerate(zip(alone, mix)):
        assert same_results(b, a), f"request {i}: " + first_mismatch(b, a)


def test_serve_admission_refuses_what_the_pool_cannot_hold(cuda):
    """A tiny pool: a request whose puts could need more slabs than are free
    completes with LSB_ERR_OOM and no effect; reads still run; the device
    never raises OOM."""
    m = Map(1, pool_slabs=4, max_window=1 << 14)
    srv = Server(m, max_wave_ops=1 << 12, ring_requests=64, arena_ops=1 << 14)
    srv.start()
    keys = W.prefill_keys(7, 2000)
    big_put = (np.full(2000, OP_PUT, np.uint8), keys, keys)
    small_put = (np.full(2, OP_PUT, np.uint8), keys[:2], keys[:2])
    gets = (np.zeros(3, np.uint8), keys[:3], np.zeros(3, np.uint64))
    reqs = [small_put, big_put, gets]
    tk = _submit_all(srv, reqs)
    res, st = _take_all(srv, reqs, tk)
    srv.stop()
    srv.close()
    assert st == [0, _lib.LSB_ERR_OOM, 0]
    assert res[2]["found"].tolist() == [1, 1, 0]
    assert res[2]["value"][:2].tolist() == keys[:2].tolist()
    k, _ = m.dump()
    assert sorted(k.tolist()) == sorted(keys[:2].tolist())
    assert m.status() == 0


def test_serve_open_loop_generator(cuda):
    """The C++ open-loop generator: Poisson arrivals over a pool of requests;
    every result equals the replay of the issued sequence."""
    pool = _requests(9, 40, 300, key_space=200)
    pool_n = np.array([len(r[1]) for r in pool], np.uint32)
    pool_off = np.concatenate([[0], np.cumsum(pool_n)[:-1]]).astype(np.uint64)
    t = np.concatenate([r[0] for r in pool])
    k = np.concatenate([r[1] for r in pool])
    v = np.concatenate([r[2] for r in pool])
    rng = np.random.default_rng(1)
    nreq = 400
    idx = rng.integers(0, len(pool), size=nreq).astype(np.uint32)
    arrival = np.cumsum(rng.exponential(20_000.0, size=nreq)).astype(np.uint64)  # ~50k req/s
    m = Map(8, max_window=1 << 16)
    srv = Server(m, max_wave_ops=1 << 14, ring_requests=256, arena_ops=1 << 16)
    srv.start()
    q0 = srv.query()
    lat, wall, res = srv.run_load(arrival, idx, pool_off, pool_n, t, k, v, want_results=True)
    q1 = srv.query()
    stats = srv.stop()
    srv.close()
    assert stats["requests"] == nreq
    assert (lat > 0).all() and wall > 0
    # the loop's step times (lsb_serve_query): every wave has gather, engine
    # and tail time, the sums only grow, and stop reports at least as much
    assert q1["waves"] > q0["waves"] and q1["requests"] == nreq
    for key in ("gather_ns", "engine_ns", "tail_ns"):
        assert q1[key] > q0[key], key
        assert stats[key] >= q1[key], key
    # the three steps of the waves fit inside the run's wall time
    busy = sum(q1[key] - q0[key] for key in ("gather_ns", "engine_ns", "tail_ns"))
    assert busy <= wall * 1.05 + 1_000_000
    seq = [slice(int(pool_off[i]), int(pool_off[i]) + int(pool_n[i])) for i in idx]
    want = OracleMap(8).mixed(np.concatenate([t[s] for s in seq]), np.concatenate([k[s] for s in seq]),
                              np.concatenate([v[s] for s in seq]))
    assert same_results(res, want), first_mismatch(res, want)
    assert m.status() == 0


def test_serve_ends_after_idle_limit(cuda):
    m = Map(4)
    srv = Server(m, idle_ms=50)
    srv.start()
    tk = srv.submit(None, np.arange(5, dtype=np.uint64))
    time.sleep(1.0)
    assert srv.done(tk)
    stats = srv.stop()
    srv.close()
    assert stats["state"] == 3 and stats["requests"] == 1
    assert m.status() == 0


def test_serve_small_arena_wraps_many_laps(cuda):
    """An arena of 4096 ops and requests of up to 600: requests skip to the
    next lap instead of wrapping, waves stop at a lap boundary, and slots are
    reused many times; results still equal the replay."""
    pool = _requests(13, 64, 600, key_space=300)
    pool_n = np.array([len(r[1]) for r in pool], np.uint32)
    pool_off = np.concatenate([[0], np.cumsum(pool_n)[:-1]]).astype(np.uint64)
    t = np.concatenate([r[0] for r in pool])
    k = np.concatenate([r[1] for r in pool])
    v = np.concatenate([r[2] for r in pool])
    rng = np.random.default_rng(2)
    nreq = 600
    idx = rng.integers(0, len(pool), size=nreq).astype(np.uint32)
    arrival = np.zeros(nreq, np.uint64)  # all due at once: the queue stays full
    m = Map(8, max_window=1 << 14)
    srv = Server(m, max_wave_ops=1 << 12, ring_requests=32, arena_ops=1 << 12)
    srv.start()
    lat, wall, res = srv.run_load(arrival, idx, pool_off, pool_n, t, k, v, want_results=True)
    stats = srv.stop()
    srv.close()
    assert stats["requests"] == nreq and stats["ops"] == int(pool_n[idx].sum())
    seq = [slice(int(pool_off[i]), int(pool_off[i]) + int(pool_n[i])) for i in idx]
    want = OracleMap(8).mixed(np.concatenate([t[s] for s in seq]), np.concatenate([k[s] for s in seq]),
                              np.concatenate([v[s] for s in seq]))
    assert same_results(res, want), first_mismatch(res, want)
    assert m.status() == 0


def test_serve_wave_stops_at_lap_boundary(cuda):
    """A request that ends exactly at the end of the arena's lap, queued
    together with one that starts the next lap: they run as separate waves (a
    wave's ops never wrap the arena), and results equal the replay."""
    rng = np.random.default_rng(21)
    sizes = (1000, 1048, 500)  # the second ends at op 2048 = the lap's end
    reqs = []
    for n in sizes:
        t = rng.choice([OP_GET, OP_PUT, OP_REMOVE], size=n, p=[0.4, 0.4, 0.2]).astype(np.uint8)
        k = W.key_of_rank(21, rng.integers(0, 300, size=n).astype(np.uint64))
        v = rng.integers(0, 2**63, size=n, dtype=np.int64).astype(np.uint64)
        reqs.append((t, k, v))
    m = Map(8, max_window=1 << 14)
    srv = Server(m, max_wave_ops=2048, ring_requests=16, arena_ops=2048)
    srv.start()
    got0, st0 = _take_all(srv, reqs[:1], _submit_all(srv, reqs[:1]))
    first = srv.stop()
    # queued while the loop is stopped, so one admission sees both
    tk = _submit_all(srv, reqs[1:])
    srv.start()
    got, st = _take_all(srv, reqs[1:], tk)
    stats = srv.stop()
    srv.close()
    assert st0 == [0] and st == [0, 0]
    assert stats["waves"] - first["waves"] == 2, "the two requests shared a wave across the lap"
    want = OracleMap(8).mixed(np.concatenate([r[0] for r in reqs]),
                              np.concatenate([r[1] for r in reqs]),
                              np.concatenate([r[2] for r in reqs]))
    g = np.concatenate(got0 + got)
    assert same_results(g, want), first_mismatch(g, want)
    assert m.status() == 0


def _mix64(k: np.ndarray) -> np.ndarray:
    """MurmurHash3's 64-bit finaliser, the library's bucket hash."""
    k = k.astype(np.uint64).copy()
    with np.errstate(over="ignore"):
        k ^= k >> np.uint64(33)
        k *= np.uint64(0xFF51AFD7ED558CCD)
        k ^= k >> np.uint64(33)
        k *= np.uint64(0xC4CEB9FE1A85EC53)
        k ^= k >> np.uint64(33)
    return k


def test_serve_admission_counts_slabs_left_in_sm_ranges(cuda):
    """A pool large enough for 32-slab per-SM refills, filled until the global
    cursor is spent while SM ranges still hold unused slabs: a put request
    that fits those slabs is admitted (not refused) and runs without a device
    OOM, and results equal the replay."""
    log2, cap = 10, 40000  # cap / (8 * 148 SMs) >= 32: full-size refills; chains ~40 slabs
    m = Map(log2, pool_slabs=cap, max_window=1 << 16)
    mask = np.uint64((1 << log2) - 1)
    keys = W.prefill_keys(31, 28 * (cap + (1 << log2)))
    o = OracleMap(log2, 2 * cap)
    placed = 0
    for step in (1 << 16, 1 << 14, 1 << 12):
        while placed + step <= len(keys) and m.pool_usage()[0] < cap:
            b = keys[placed:placed + step]
            cnt = np.bincount((_mix64(keys[:placed + step]) & mask).astype(np.int64),
                              minlength=1 << log2)
            linked = int(np.maximum(0, (cnt + 27) // 28 - 1).sum())
            if linked > cap - 800:
                break
            m.put(dev(b), dev(b))
            o.put(b, b)
            placed += step
    used, _ = m.pool_usage()
    cnt = np.bincount((_mix64(keys[:placed]) & mask).astype(np.int64), minlength=1 << log2)
    linked = int(np.maximum(0, (cnt + 27) // 28 - 1).sum())
    assert m.status() == 0
    assert used == cap, f"cursor not spent ({used} of {cap}); the case is not reached"
    left = cap - linked
    assert left >= 500, left
    new = W.prefill_keys(32, 400)
    req = (np.full(400, OP_PUT, np.uint8), new, new)
    srv = Server(m, max_wave_ops=1 << 12, ring_requests=16, arena_ops=1 << 14)
    srv.start()
    res, st = _take_all(srv, [req], _submit_all(srv, [req]))
    srv.stop()
    srv.close()
    assert st == [0], "refused although the SM ranges hold enough slabs"
    assert m.status() == 0
    want = o.mixed(req[0], req[1], req[2])
    assert same_results(res[0], want), first_mismatch(res[0], want)
    assert m.size() == placed + 400
