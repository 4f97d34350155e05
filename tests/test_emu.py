"""CPU checks of the library's own device code under a host emulation of the
CUDA execution model (tests/emu/simt_host.h): each CUDA thread is a host
thread, each grid step runs all of its blocks before the next.

The window-ordering phase (group formation, per-group ordering including the
multi-step path for groups of more than 4096 members) is checked against the
index order it must produce; the whole per-phase batch (probe, ordering,
resolve) is built with AddressSanitizer, so every access of those phases is
checked against its buffer, and its results are compared with the oracle.
The serving loop's gather is checked on every source alignment."""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from lslab_b200 import workload as W
from oracle import OracleMap

ROOT = Path(__file__).resolve().parents[1]
EMU = ROOT / "tests" / "emu"
CSRC = ROOT / "lslab_b200" / "csrc"

pytestmark = pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")


def _build(out: Path, src: str, sanitize: bool) -> Path:
    cmd = ["g++", "-std=c++20", "-O1", "-g", "-pthread", "-DLSB_HOST_EMU", f"-I{EMU}",
           f"-I{CSRC}", str(EMU / src), "-o", str(out)]
    if sanitize:
        cmd[1:1] = ["-fsanitize=address", "-fno-omit-frame-pointer"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return out


@pytest.fixture(scope="module")
def bins(tmp_path_factory):
    d = tmp_path_factory.mktemp("emu")
    return {"order": _build(d / "order_emu", "order_emu.cpp", False),
            "window": _build(d / "window_emu", "window_emu.cpp", True)}


def _write_window(path: Path, types, keys, window, vals=None):
    with open(path, "wb") as f:
        f.write(np.array([len(keys), window], np.uint32).tobytes())
        f.write(np.asarray(types, np.uint8).tobytes())
        f.write(np.asarray(keys, np.uint64).tobytes())
        if vals is not None:
            f.write(np.asarray(vals, np.uint64).tobytes())


def _order_cases():
    rng = np.random.default_rng(5)
    out = {}
    n = 60_000  # one key carries half the ops: ~12k mutations in one group
    t = rng.choice([0, 1, 2], size=n, p=[0.6, 0.3, 0.1]).astype(np.uint8)
    k = W.key_of_rank(9, rng.integers(0, 40, size=n))
    k[rng.random(n) < 0.5] = np.uint64(0xDEADBEEF)
    out["hot"] = (t, k, 1 << 17)
    n = 20_000  # every op a put of one key
    out["one_key"] = (np.ones(n, np.uint8), np.full(n, 42, np.uint64), 1 << 15)
    n = 10_001  # exactly 4097 members, window not a multiple of the range count
    t = np.zeros(n, np.uint8)
    k = W.key_of_rank(1, np.arange(n) % 97)
    idx = np.sort(rng.choice(n, 4097, replace=False))
    t[idx], k[idx] = 1, 5
    out["just_over"] = (t, k, n)
    n = 1 << 16  # a dense block of one key, a few strays far away, two more hot keys
    t = rng.choice([0, 1, 2], size=n, p=[0.3, 0.5, 0.2]).astype(np.uint8)
    k = W.key_of_rank(3, rng.integers(0, 3000, size=n))
    k[30_000:40_000] = 8
    k[rng.integers(0, n, size=20)] = 8
    k[rng.random(n) < 0.15] = 9
    k[rng.random(n) < 0.1] = 10
    out["dense_and_strays"] = (t, k, 1 << 16)
    return out


ORDER = _order_cases()


@pytest.mark.parametrize("case", sorted(ORDER))
@pytest.mark.parametrize("threads,blocks", [(256, 3), (512, 2)])
def test_ordering_matches_index_order(bins, tmp_path, case, threads, blocks):
    t, k, window = ORDER[case]
    path = tmp_path / "w.bin"
    _write_window(path, t, k, window)
    r = subprocess.run([str(bins["order"]), str(path), str(threads), str(blocks), "7"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.startswith("OK"), r.stdout + r.stderr


@pytest.mark.parametrize("mode,window", [("tiles", 16_384), ("muts_first", 16_383),
                                         ("muts_first_binned", 16_384)])
def test_whole_batch_in_bounds_and_equal_to_oracle(bins, tmp_path, mode, window):
    """Probe, ordering (with a group of ~5k mutations) and resolve of a mixed
    batch over two windows, under AddressSanitizer.  muts_first probes the way
    the fused kernel's split-0 form does (mutation list, then the reads);
    muts_first_binned probes the reads in table-region order.  The
    muts_first window size puts the second window's types off 16-byte
    alignment and ends the first with a partial span."""
    n, log2 = 24_000, 6
    rng = np.random.default_rng(11)
    t = rng.choice([0, 1, 2], size=n, p=[0.5, 0.35, 0.15]).astype(np.uint8)
    k = W.key_of_rank(2, rng.integers(0, 400, size=n))
    k[rng.random(n) < 0.45] = np.uint64(77)
    v = W.splitmix64(13, 0, n)
    path, outp = tmp_path / "ops.bin", tmp_path / "out.bin"
    _write_window(path, t, k, window, v)
    want = OracleMap(log2).mixed(t, k, v)
    pool = (1 << log2) // 4 + 4096
    r = subprocess.run([str(bins["window"]), str(path), str(log2), str(pool), "256", str(outp)]
                       + ([mode] if mode != "tiles" else []),
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr[-4000:]
    raw = np.fromfile(outp, np.uint8)
    got = raw[: 16 * n].view(np.dtype([("found", "u1"), ("pad", "u1", (7,)), ("value", "<u8")]))
    status = int(raw[16 * n:].view(np.uint32)[0])
    assert status == 0
    bad = np.nonzero((got["found"] != want["found"]) | (got["value"] != want["value"]))[0]
    assert bad.size == 0, f"{bad.size} mismatches, first at {bad[:5]}"


def _update_case(kind: str):
    """Mixed batches with updates (update-if-present): whether an update
    takes effect depends on the last earlier put or remove of its key in the
    batch, so groups of every ordering path are covered: inline (<= 8
    members), warp (<= 64), block (<= 4096) and hot keys over several runs."""
    n = 10_000
    rng = np.random.default_rng(17)
    if kind == "mixed":
        t = rng.choice([0, 1, 2, 3], size=n, p=[0.4, 0.2, 0.15, 0.25]).astype(np.uint8)
        k = W.key_of_rank(4, rng.integers(0, 400, size=n))
        k[rng.random(n) < 0.45] = np.uint64(77)  # ~2.7k mutations of one key
    else:  # "update_runs": a hot key whose ops are nearly all updates, with
        # rare puts and removes, so whole runs of its members carry nothing
        t = np.full(n, 3, np.uint8)
        t[rng.random(n) < 0.004] = 1
        t[rng.random(n) < 0.003] = 2
        t[rng.random(n) < 0.2] = 0
        k = W.key_of_rank(6, rng.integers(0, 50, size=n))
        k[rng.random(n) < 0.7] = np.uint64(91)
    v = W.splitmix64(19, 0, n)
    return t, k, v


@pytest.mark.parametrize("kind,mode,window", [("mixed", "tiles", 16_384),
                                               ("mixed", "muts_first", 16_383),
                                               ("update_runs", "tiles", 16_384)])
def test_updates_in_bounds_and_equal_to_oracle(bins, tmp_path, kind, mode, window):
    t, k, v = _update_case(kind)
    log2 = 6
    # half of the keys present before the batch: updates of them take effect
    pre = np.unique(k)[::2]
    o = OracleMap(log2)
    o.put(pre, pre ^ np.uint64(5))
    want = o.mixed(t, k, v)
    tt = np.concatenate([np.ones(len(pre), np.uint8), t])
    kk = np.concatenate([pre, k])
    vv = np.concatenate([pre ^ np.uint64(5), v])
    path, outp = tmp_path / "ops.bin", tmp_path / "out.bin"
    _write_window(path, tt, kk, window, vv)
    pool = (1 << log2) // 4 + 4096
    r = subprocess.run([str(bins["window"]), str(path), str(log2), str(pool), "256", str(outp)]
                       + ([mode] if mode != "tiles" else []),
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr[-4000:]
    raw = np.fromfile(outp, np.uint8)
    got = raw[: 16 * len(kk)].view(np.dtype([("found", "u1"), ("pad", "u1", (7,)), ("value", "<u8")]))
    got = got[len(pre):]
    status = int(raw[16 * len(kk):16 * len(kk) + 4].view(np.uint32)[0])
    assert status == 0
    bad = np.nonzero((got["found"] != want["found"]) | (got["value"] != want["value"]))[0]
    assert bad.size == 0, f"{bad.size} mismatches, first at {bad[:5]}"


def test_compaction_between_windows_in_bounds_and_reclaims(bins, tmp_path):
    """Put/remove churn at a roughly constant live count over many windows,
    with every chain compacted after each window: results equal the oracle
    (compaction moves entries but changes no contents), no access leaves its
    buffer, and the slabs the churn needs come back from the free stack (the
    bump cursor stays far below what 8 windows of fresh keys would take)."""
    log2, window, nwin, per = 5, 2048, 8, 700
    rng = np.random.default_rng(23)
    t_all, k_all = [], []
    for w in range(nwin):
        new = W.prefill_keys(40 + w, per)  # fresh keys each window
        old = W.prefill_keys(40 + w - 2, per) if w >= 2 else np.zeros(0, np.uint64)
        ks = np.concatenate([new, old, W.prefill_keys(40 + max(0, w - 1), 500)])
        ts = np.concatenate([np.ones(per, np.uint8), np.full(len(old), 2, np.uint8),
                             np.zeros(500, np.uint8)])
        o = rng.permutation(len(ks))[:window]
        t_all.append(ts[o])
        k_all.append(ks[o])
    t = np.concatenate(t_all)
    k = np.concatenate(k_all)
    v = W.splitmix64(29, 0, len(k))
    path, outp = tmp_path / "ops.bin", tmp_path / "out.bin"
    _write_window(path, t, k, window, v)
    want = OracleMap(log2).mixed(t, k, v)
    pool = 8192
    r = subprocess.run([str(bins["window"]), str(path), str(log2), str(pool), "256", str(outp),
                        "compact"], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr[-4000:]
    raw = np.fromfile(outp, np.uint8)
    n = len(k)
    got = raw[: 16 * n].view(np.dtype([("found", "u1"), ("pad", "u1", (7,)), ("value", "<u8")]))
    status = int(raw[16 * n:16 * n + 4].view(np.uint32)[0])
    cursor, top = raw[16 * n + 4:16 * n + 20].view(np.uint64).tolist()
    assert status == 0
    bad = np.nonzero((got["found"] != want["found"]) | (got["value"] != want["value"]))[0]
    assert bad.size == 0, f"{bad.size} mismatches, first at {bad[:5]}"
    inserted = int((t == 1).sum())
    bumped = cursor - (1 << log2)
    # fresh slabs bumped stay well below one slab per 28 inserts of the whole
    # run, and the last compaction left emptied slabs on the free stack
    assert bumped < inserted // 28 // 2, (bumped, inserted)
    assert top > 0, top


def test_lock_free_inserts_race_without_losing_keys_or_slabs(bins, tmp_path):
    """LSB_LOCK_FREE writers (CAS on tag and link words) inserting thousands
    of distinct keys into 8 buckets in one window, on concurrent host
    threads: every key lands (results and a later read equal the oracle),
    and chains grow by about one slab per 28 keys (a thread that loses a
    link race keeps its slab and appends it instead of dropping it)."""
    log2, n = 3, 6000
    keys = W.prefill_keys(61, n)
    t = np.concatenate([np.ones(n, np.uint8), np.zeros(n, np.uint8)])
    k = np.concatenate([keys, keys])
    v = np.concatenate([keys ^ np.uint64(9), np.zeros(n, np.uint64)])
    window = n  # the inserts in one window, the reads in the next
    path, outp = tmp_path / "ops.bin", tmp_path / "out.bin"
    _write_window(path, t, k, window, v)
    want = OracleMap(log2).mixed(t, k, v)
    pool = 4096
    r = subprocess.run([str(bins["window"]), str(path), str(log2), str(pool), "256", str(outp),
                        "lockfree"], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr[-4000:]
    raw = np.fromfile(outp, np.uint8)
    m = len(k)
    got = raw[: 16 * m].view(np.dtype([("found", "u1"), ("pad", "u1", (7,)), ("value", "<u8")]))
    status = int(raw[16 * m:16 * m + 4].view(np.uint32)[0])
    cursor = int(raw[16 * m + 4:16 * m + 12].view(np.uint64)[0])
    assert status == 0
    bad = np.nonzero((got["found"] != want["found"]) | (got["value"] != want["value"]))[0]
    assert bad.size == 0, f"{bad.size} mismatches, first at {bad[:5]}"
    needed = n // 28 - (1 << log2)  # overflow slabs of perfectly packed chains
    assert cursor - (1 << log2) <= needed + 2 * (1 << log2) + 64, (cursor, needed)


def test_v32_put_batch_equals_oracle(bins, tmp_path):
    """A put batch with 32-bit values and 32-bit old values out (the window
    lsb_map_put_v32 runs), keys repeated across the batch: every old value
    equals the oracle's."""
    rng = np.random.default_rng(32)
    n, log2 = 12_000, 6
    k = W.key_of_rank(32, rng.integers(0, 4000, size=n).astype(np.uint64))
    v = rng.integers(0, 2**32, size=n, dtype=np.uint64)
    path, outp = tmp_path / "ops.bin", tmp_path / "out.bin"
    _write_window(path, np.ones(n, np.uint8), k, 16_384, v)
    want = OracleMap(log2).put(k, v)
    pool = (1 << log2) // 4 + 4096
    r = subprocess.run([str(bins["window"]), str(path), str(log2), str(pool), "256", str(outp),
                        "v32put"], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout + r.stderr[-4000:]
    raw = np.fromfile(outp, np.uint8)
    got = raw[: 4 * n].view(np.uint32)
    status = int(raw[4 * n:4 * n + 4].view(np.uint32)[0])
    assert status == 0
    bad = np.nonzero(got != want.astype(np.uint32))[0]
    assert bad.size == 0, f"{bad.size} mismatches, first at {bad[:5]}: {got[bad[:3]]} vs {want[bad[:3]]}"


def test_serving_gather_covers_every_alignment(tmp_path):
    """The serving loop's gather (lsb_gather.cuh, host build under
    AddressSanitizer): for source offsets 0..31 bytes, 0..200 ops and 1..151
    threads, the threads together copy the ops exactly once, write nothing
    past them, read nothing outside them, and load 16 bytes only at aligned
    addresses."""
    exe = _build(tmp_path / "gather_emu", "gather_emu.cpp", True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr[-2000:]
