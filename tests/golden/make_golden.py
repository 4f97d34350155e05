"""Generate golden vectors from the reference's OWN kernels.

Runs lslab::map<uint64_t,uint64_t> / lslab::set<uint32_t> (built for sm_100a
from the reference headers into oracle/_ref/liblslab_ref.so) on small seeded
inputs and stores inputs and outputs as .npz fixtures.  tests/test_oracle.py
checks the CPU oracle against them bit for bit, which pins the oracle to the
reference.  Needs a GPU; run as

    python tests/golden/make_golden.py --out tests/golden

Every case is free of cross-warp same-key conflicts (where the reference's
answer is unique); same-key ops inside one warp are kept on purpose, the
reference orders them by lane.
"""
from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from lslab_b200 import workload as W  # noqa: E402
from oracle import RefMap, RefSet, ref_map_pool_bound  # noqa: E402


def _dev(a):
    import torch
    a = np.ascontiguousarray(a)
    view = {np.dtype(np.uint64): np.int64, np.dtype(np.uint32): np.int32}.get(a.dtype, a.dtype)
    return torch.from_numpy(a.view(view).copy()).cuda()


def _host(t, dtype):
    return t.cpu().numpy().view(dtype).reshape(-1)


def _res(n):
    import torch
    return torch.zeros((n, 2), dtype=torch.int64, device="cuda")


def _split(r):
    b = r.cpu().numpy().reshape(-1, 2)
    return (b[:, 0].view(np.uint64) & np.uint64(0xFF)).astype(np.uint8), b[:, 1].view(np.uint64)


def map_gets(out: Path):
    import torch
    seed, log2, n = 1001, 10, 1 << 13
    pk = W.prefill_keys(seed, n)
    pv = W.prefill_values(pk)
    ak = W.absent_keys(seed, n, pk)
    q = np.concatenate([pk[: n // 2], ak[: n // 2]])
    q = q[np.argsort(W.splitmix64(seed + 5, 0, len(q)))]
    m = RefMap(log2, ref_map_pool_bound(log2, pk))
    old = torch.zeros(n, dtype=torch.int64, device="cuda")
    m.put(_dev(pk), _dev(pv), old)
    r = _res(len(q))
    m.get(_dev(q), r)
    torch.cuda.synchronize()
    f, v = _split(r)
    v = np.where(f == 1, v, np.uint64(0))  # .second is unwritten on a miss
    dk, dv = m.dump()
    np.savez_compressed(out / "map_gets.npz", log2=log2, put_keys=pk, put_vals=pv,
                        put_old=_host(old, np.uint64), get_keys=q, get_found=f, get_value=v,
                        dump_keys=dk, dump_vals=dv, pool_used=m.pool_used())


def map_put_remove(out: Path):
    import torch
    seed, log2 = 1002, 6
    base = W.prefill_keys(seed, 6000)
    m = RefMap(log2, ref_map_pool_bound(log2, np.concatenate([base, base])))
    rec = {"log2": log2}
    steps = [("put", base[:2000]), ("put", base[1000:4000]), ("put", base[3000:6000]),
             ("remove", base[::3]), ("put", base[::6]), ("get", base[::2])]
    for i, (kind, keys) in enumerate(steps):
        rec[f"s{i}_kind"] = kind
        rec[f"s{i}_keys"] = keys
        if kind == "put":
            vals = W.splitmix64(seed + 10 + i, 0, len(keys))
            old = torch.zeros(len(keys), dtype=torch.int64, device="cuda")
            m.put(_dev(keys), _dev(vals), old)
            torch.cuda.synchronize()
            rec[f"s{i}_vals"] = vals
            rec[f"s{i}_old"] = _host(old, np.uint64)
        else:
            r = _res(len(keys))
            (m.remove if kind == "remove" else m.get)(_dev(keys), r)
            torch.cuda.synchronize()
            f, v = _split(r)
            rec[f"s{i}_found"] = f
            rec[f"s{i}_value"] = np.where(f == 1, v, np.uint64(0))
    rec["dump_keys"], rec["dump_vals"] = m.dump()
    rec["steps"] = len(steps)
    np.savez_compressed(out / "map_put_remove.npz", **rec)


def map_warp_chain(out: Path):
    import torch
    keys = np.full(32, 0x1234, np.uint64)
    vals = np.arange(100, 132, dtype=np.uint64)
    m = RefMap(4, 16)
    old = torch.zeros(32, dtype=torch.int64, device="cuda")
    m.put(_dev(keys), _dev(vals), old)
    torch.cuda.synchronize()
    np.savez_compressed(out / "map_warp_chain.npz", keys=keys, vals=vals,
                        old=_host(old, np.uint64))


def set_batches(out: Path):
    import torch
    seed, log2 = 1003, 7
    pre = W.set_prefill_keys(seed, 31 * (1 << log2))
    batches = [W.set_mixed_batch(seed, b, 1 << 11) for b in range(4)]
    inserts = np.concatenate([pre] + [bt.keys[bt.types == 1] for bt in batches])
    s = RefSet(log2, ref_map_pool_bound(log2, inserts.astype(np.uint64)))
    r = torch.zeros(len(pre), dtype=torch.uint8, device="cuda")
    s.insert(_dev(pre), r)
    rec = {"log2": log2, "pre": pre}
    step = 0
    for b, bt in enumerate(batches):
        for t, name in ((0, "contains"), (1, "insert"), (2, "remove")):
            k = np.unique(bt.keys[bt.types == t])
            k = k[np.argsort(W.splitmix64(seed + 7 * b + t, 0, len(k)))]
            o = torch.zeros(len(k), dtype=torch.uint8, device="cuda")
            getattr(s, name)(_dev(k), o)
            torch.cuda.synchronize()
            rec[f"s{step}_kind"] = name
            rec[f"s{step}_keys"] = k
            rec[f"s{step}_out"] = _host(o, np.uint8)
            step += 1
    rec["steps"] = step
    rec["dump"] = s.dump()
    np.savez_compressed(out / "set_batches.npz", **rec)


def set_known_answer(out: Path):
    import torch
    s = RefSet(10, 64)
    keys = np.arange(1, 1025, dtype=np.uint32)
    outs = []
    for rep in range(3):
        for name in ("insert", "contains", "remove", "contains"):
            o = torch.zeros(1024, dtype=torch.uint8, device="cuda")
            getattr(s, name)(_dev(keys), o)
            torch.cuda.synchronize()
            outs.append(_host(o, np.uint8))
    np.savez_compressed(out / "set_known_answer.npz", keys=keys, outs=np.stack(outs))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(Path(__file__).resolve().parent))
    a = ap.parse_args()
    out = Path(a.out)
    out.mkdir(parents=True, exist_ok=True)
    for f in (map_gets, map_put_remove, map_warp_chain, set_batches, set_known_answer):
        f(out)
        print("wrote", f.__name__)


if __name__ == "__main__":
    main()
