"""Benchmark: batched get/put on map<uint64,uint64>, the headline workload.

Workload (default): map with 2^22 buckets (table > L2), prefilled with 2^26
splitmix64 keys (value = key ^ 0x9E3779B97F4A7C15); each step is one batch of
2^20 ops, 95% get / 5% put, keys Zipf(0.99) over the 2^26 prefill keys, put
values uniform u64; a batch is issued gets first, then puts (the order a
per-op-type caller issues it).  Synthetic seeded data; every step uses a
distinct batch.

Arms:
  ours (default)   `value`: the fused persistent kernel (lsb_map_execute_fused)
                   draining the queue of timed batches in one launch, launch
                   shape chosen by the autotuner on a warm-up batch, inputs
                   resident in HBM; `per_batch_launch_value`: the same kernel
                   one launch per batch; `plain_value`: per-op-type launches
                   (lsb_map_get then lsb_map_put) on an identical table, results
                   checked bit-identical to the fused path; `e2e`: the fused call
                   with pinned HOST buffers, H2D of the batch and D2H of the
                   results inside the timed region, consecutive batches
                   pipelined over a copy-in stream, the compute stream and a
                   copy-out stream.
  --impl reference lslab's own kernels (map::get / map::put, built for sm_100a
                   from the reference sources into oracle/_ref) on the same
                   workload, per-op-type launches as the reference's API offers.

Multi-GPU (torchrun, one rank per GPU): every rank owns an independent table
shard and its own batch stream (weak scaling, no data-path collective); time is
the max over ranks of the device-timed region.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mops/s (95/5 get/put, Zipf 0.99) batched vs plain kernels; p50/p99 latency"
BYTES_GET = 88   # request 8 + response 16 + key sector 32 + value sector 32
BYTES_PUT = 120  # request 16 + response 8 + key sector 32 + value sector 32 + write-back 32


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="zipf9505",
                    choices=["zipf9505", "batches", "serving", "sets", "locks", "plain-small",
                             "probes"],
                    help="zipf9505: the headline line; batches: 4096 uneven mixed batches in "
                         "one graph-captured fused launch vs per-op-type calls; serving: the "
                         "request loop under open-loop Poisson load")
    ap.add_argument("--wave-ops", type=int, default=1 << 16, help="serving: ops per wave")
    ap.add_argument("--serve-seconds", type=float, default=1.0,
                    help="serving: offered-load duration of each sweep point")
    ap.add_argument("--serve-loads", default="0.1,0.3,0.5,0.7,0.9,1.0",
                    help="serving: offered loads as fractions of the measured peak")
    ap.add_argument("--nbatches", type=int, default=4096)
    ap.add_argument("--set-log2", default="18,24", help="sets: table sizes (log2 buckets)")
    ap.add_argument("--set-lf", default="0.25,0.5,1,2,4", help="sets: keys per head-slab slot")
    ap.add_argument("--set-forms", default="fused,plain,lslab", help="sets: forms to run")
    ap.add_argument("--no-autotune", action="store_true",
                    help="zipf9505 and batches: library-default (or --block/--chunk/...) "
                         "tuning instead of the autotuner")
    ap.add_argument("--buckets-log2", type=int, default=22)
    ap.add_argument("--prefill-log2", type=int, default=26)
    ap.add_argument("--batch-log2", type=int, default=20)
    ap.add_argument("--theta", type=float, default=0.99)
    ap.add_argument("--put-frac", type=float, default=0.05)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--soak-s", type=float, default=1.0,
                    help="untimed read-only load before timing so clocks leave idle")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-side", action="store_true",
                    help="headline run: skip the side workloads (plain-small against lslab, "
                         "uneven batches, serving) whose summaries the line carries")
    ap.add_argument("--cpu-batches", type=int, default=4)
    ap.add_argument("--cpu-seconds", type=float, default=3.0)
    ap.add_argument("--lock-mode", default="writer", choices=["writer", "free", "rw"])
    ap.add_argument("--block", type=int, default=0, help="threads per block (0 = library default)")
    ap.add_argument("--prefetch", type=int, default=-1)
    ap.add_argument("--chunk", type=int, default=-1)
    ap.add_argument("--dedup", type=int, default=-1)
    ap.add_argument("--split", type=int, default=-1, help="fused: percent of reads probed first")
    ap.add_argument("--region", type=int, default=-1, help="fused: probe in table-region order")
    ap.add_argument("--read-order", type=int, default=-1,
                    help="read calls: 0 op order, 1 table-region order")
    ap.add_argument("--overlap", type=int, default=-1,
                    help="batched calls: 1 = reads in the lean read kernel beside the mutation "
                         "steps on a second stream")
    ap.add_argument("--trace", action="store_true", help="single mode: print fused phase times")
    ap.add_argument("--single", action="store_true",
                    help="fused timing only (one table, no plain/e2e/cpu legs): the small "
                         "case for profiler captures")
    ap.add_argument("--plain", action="store_true",
                    help="with --single: time the per-op-type calls (a get call and a put "
                         "call per batch) instead of the fused kernel")
    return ap.parse_args()


# ------------------------------------------------------------------ helpers
class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons while running."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,utilization.gpu,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(index)], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = []
        for line in Path(self.f.name).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[0]), float(parts[1]), float(parts[3]), parts[5:9]))
            except ValueError:
                continue
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        loaded = [r for r in rows if r[2] > 0] or rows
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[j] for r in loaded for j, v in enumerate(r[3]) if v == "Active"})
        return {"sm_mhz": statistics.median(r[0] for r in loaded), "sm_max_mhz": rows[0][1],
                "reasons": reasons, "samples": len(rows), "samples_under_load": len(loaded)}


def dev_u64(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(name: str):
    """Per-launch DRAM bytes of the dominant kernel from the committed ncu
    summary (profiles/<name>.txt, line 'dram_bytes_per_launch: N'), or None."""
    p = ROOT / "profiles" / f"{name}.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("dram_bytes_per_launch:"):
            return float(line.split(":", 1)[1])
    return None


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def max_over_ranks(x: float, world: int) -> float:
    from lslab_b200.shard import max_over_ranks as mor
    return mor(x) if world > 1 else x


def barrier(world: int):
    if world > 1:
        from lslab_b200.shard import barrier as b
        b()


# ------------------------------------------------------------------ workload
def make_batches(args, rank: int, count: int):
    from lslab_b200 import workload as W
    from lslab_b200.shard import rank_seed
    seed = rank_seed(args.seed, rank)
    n = 1 << args.batch_log2
    items = 1 << args.prefill_log2
    return [W.map_zipf_batch(seed, b, n, items, args.theta, (1 - args.put_frac, args.put_frac))
            for b in range(count)]


def prefill_arrays(args, rank: int):
    from lslab_b200 import workload as W
    from lslab_b200.shard import rank_seed
    seed = rank_seed(args.seed, rank)
    keys = W.prefill_keys(seed, 1 << args.prefill_log2)
    return keys, W.prefill_values(keys)


def alg_bytes(batch) -> float:
    nput = int(np.sum(batch.types == 1))
    return (len(batch.keys) - nput) * BYTES_GET + nput * BYTES_PUT


def apply_tuning(args, table):
    kw = {}
    if args.block:
        kw["block_threads"] = args.block
    if args.prefetch >= 0:
        kw["prefetch"] = args.prefetch
    if args.chunk >= 0:
        kw["chunk"] = args.chunk
    if args.dedup >= 0:
        kw["dedup"] = args.dedup
    if args.split >= 0:
        kw["fused_split"] = args.split
    if args.region >= 0:
        kw["region_order"] = args.region
    if args.overlap >= 0:
        kw["overlap"] = args.overlap
    if args.read_order >= 0:
        kw["read_order"] = args.read_order
    if kw:
        table.set_tuning(**kw)


# ------------------------------------------------------------------ our arm
def run_ours(args, world, rank, local):
    import torch
    import lslab_b200 as L

    stream = torch.cuda.current_stream()
    n = 1 << args.batch_log2
    nb = args.warmup + args.steps
    batches = make_batches(args, rank, nb)
    pk, pv = prefill_arrays(args, rank)
    pool = max(1 << (args.buckets_log2 - 2), 4096)
    fused = L.Map(args.buckets_log2, pool, lock_mode=args.lock_mode)
    plain = fused if args.single else L.Map(args.buckets_log2, pool, lock_mode=args.lock_mode)
    apply_tuning(args, fused)
    apply_tuning(args, plain)
    for off in range(0, len(pk), 1 << 24):
        k = dev_u64(torch, pk[off:off + (1 << 24)])
        v = dev_u64(torch, pv[off:off + (1 << 24)])
        fused.put(k, v)
        if not args.single:
            plain.put(k, v)
        del k, v
    torch.cuda.synchronize()
    st = fused.status() | plain.status()
    assert st == 0, f"prefill raised device status {st:#x}"

    # the batches back to back in one device queue; batch b is slice b
    q_types = torch.from_numpy(np.concatenate([b.types for b in batches])).cuda()
    q_keys = dev_u64(torch, np.concatenate([b.keys for b in batches]))
    q_vals = dev_u64(torch, np.concatenate([b.vals for b in batches]))
    q_out = torch.empty((nb * n, 2), dtype=torch.int64, device="cuda")
    d_types = [q_types[b * n:(b + 1) * n] for b in range(nb)]
    d_keys = [q_keys[b * n:(b + 1) * n] for b in range(nb)]
    d_vals = [q_vals[b * n:(b + 1) * n] for b in range(nb)]
    out_f = [q_out[b * n:(b + 1) * n] for b in range(nb)]
    n_get = [int(np.sum(b.types == 0)) for b in batches]
    if args.single:
        ops = n * args.steps
        old_p = torch.empty(n, dtype=torch.int64, device="cuda")

        def step(b):
            if args.plain:  # gets then puts: the batch's own order
                g = n_get[b]
                fused.get(d_keys[b][:g], out_f[b])
                fused.put(d_keys[b][g:], d_vals[b][g:], old_p[:n - g])
            else:
                fused.execute_fused(d_types[b], d_keys[b], d_vals[b], out_f[b])

        for b in range(args.warmup):
            step(b)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for s in range(args.steps):
            step(args.warmup + s)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        phases = trace = None
        if args.trace:
            fused.set_trace(True)
            for b in range(min(3, nb)):  # the last of three traced batches is reported
                fused.execute_fused(d_types[b], d_keys[b], d_vals[b], out_f[b])
                tr = fused.read_trace()
            phases = [round((tr[k + 1][0] - tr[k][0]) / 1e3, 2) for k in range(len(tr) - 1)]
            trace = [[round((ns - tr[0][0]) / 1e3, 2), w, ph] for ns, w, ph in tr]
        if rank == 0:
            print(json.dumps({"single": True, "phases_us": phases, "trace": trace,
                              "value": round(ops / (ms * 1e-3) / 1e6, 2),
                              "unit": "Mops/s", "ms_per_step": round(ms / args.steps, 5),
                              "tuning": fused.tuning(),
                              "device_status": fused.status()}), flush=True)
        return
    out_g = [torch.empty((n, 2), dtype=torch.int64, device="cuda") for _ in range(nb)]
    out_p = [torch.empty(n - n_get[b], dtype=torch.int64, device="cuda") for b in range(nb)]

    # the autotuner picks the fused launch shape on warm-up batch 0 (untimed;
    # the batch's net effect is one application, so the plain table applies
    # it once too and the two tables stay identical)
    explicit = (args.block or args.prefetch >= 0 or args.chunk >= 0 or args.dedup >= 0
                or args.split >= 0 or args.region >= 0 or args.overlap >= 0
                or args.read_order >= 0)
    if not args.no_autotune and not explicit:
        fused.autotune(d_types[0], d_keys[0], d_vals[0], out_f[0])
        g = n_get[0]
        plain.get(d_keys[0][:g], out_g[0])
        plain.put(d_keys[0][g:], d_vals[0][g:], out_p[0])
        torch.cuda.synchronize()

    clocks = Clocks(local)
    # soak (untimed, read-only so both tables stay identical): gets of the
    # batch keys until soak_s has passed, so clocks have left idle
    t_end = time.perf_counter() + args.soak_s
    i = 0
    while time.perf_counter() < t_end:
        fused.get(d_keys[i % nb], out_f[i % nb])
        i += 1
        if i % 50 == 0:
            torch.cuda.synchronize()
    torch.cuda.synchronize()
    # warm-up (untimed): the W warm-up batches drained by one fused launch
    W, K = args.warmup, args.steps
    fused.execute_fused(q_types[:W * n], q_keys[:W * n], q_vals[:W * n], q_out[:W * n])
    torch.cuda.synchronize()

    # ---- timed: the persistent fused kernel drains the queue of K batches
    # (one window each, applied in order) in one launch
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    barrier(world)
    torch.cuda.synchronize()
    ev[0].record(stream)
    lo, hi = W * n, (W + K) * n
    fused.execute_fused(q_types[lo:hi], q_keys[lo:hi], q_vals[lo:hi], q_out[lo:hi])
    ev[1].record(stream)
    torch.cuda.synchronize()
    barrier(world)
    queue_ms = ev[0].elapsed_time(ev[1])
    fused_ms = max_over_ranks(queue_ms, world)
    identical_q = q_out[lo:hi].clone()

    # ---- the same K batches one fused launch each (applied again to the
    # fused table; results discarded): the per-batch-launch form
    scratch = torch.empty((n, 2), dtype=torch.int64, device="cuda")
    pev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    barrier(world)
    torch.cuda.synchronize()
    pev[0].record(stream)
    for s in range(K):
        b = W + s
        fused.execute_fused(d_types[b], d_keys[b], d_vals[b], scratch)
    pev[1].record(stream)
    torch.cuda.synchronize()
    barrier(world)
    per_batch_ms = max_over_ranks(pev[0].elapsed_time(pev[1]), world)
    q_out[lo:hi].copy_(identical_q)
    del identical_q

    # ---- plain per-op-type launches on an identical table
    for b in range(args.warmup):
        g = n_get[b]
        plain.get(d_keys[b][:g], out_g[b])
        plain.put(d_keys[b][g:], d_vals[b][g:], out_p[b])
    torch.cuda.synchronize()
    pe0, pe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    pe0.record(stream)
    for s in range(args.steps):
        b = args.warmup + s
        g = n_get[b]
        plain.get(d_keys[b][:g], out_g[b])
        plain.put(d_keys[b][g:], d_vals[b][g:], out_p[b])
    pe1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    plain_ms = max_over_ranks(pe0.elapsed_time(pe1), world)

    # identical results: fused out == plain (get part, then put old values)
    identical = True
    for b in range(nb):
        g = n_get[b]
        f = out_f[b]
        if not torch.equal(f[:g], out_g[b][:g]) or not torch.equal(f[g:, 1], out_p[b]):
            identical = False
            break
    st = fused.status() | plain.status()

    # ---- random-probe ceiling: the accesses of each timed batch's gets at
    # uniformly random keys of the same table, nothing else
    # (lsb_probe_calibrate over the table's head slabs)
    view = fused.device_view()
    cal_out = torch.empty((n, 2), dtype=torch.int64, device="cuda")
    for b in range(args.warmup):
        L.probe_calibrate(view["slabs"], 1 << args.buckets_log2, 480, d_keys[b][:n_get[b]],
                          cal_out, seed=b)
    cev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    torch.cuda.synchronize()
    cev[0].record(stream)
    for s in range(args.steps):
        b = args.warmup + s
        L.probe_calibrate(view["slabs"], 1 << args.buckets_log2, 480, d_keys[b][:n_get[b]],
                          cal_out, seed=b)
    cev[1].record(stream)
    torch.cuda.synchronize()
    cal_ms = max_over_ranks(cev[0].elapsed_time(cev[1]), world)
    cal_gets = sum(n_get[args.warmup:])
    del cal_out

    # ---- e2e through the public API with host buffers
    h_types = [torch.from_numpy(b.types).pin_memory() for b in batches]
    h_keys = [torch.from_numpy(b.keys.view(np.int64)).pin_memory() for b in batches]
    h_vals = [torch.from_numpy(b.vals.view(np.int64)).pin_memory() for b in batches]
    h_out = torch.empty((n, 2), dtype=torch.int64).pin_memory()
    # Pipelined over three streams and a ring of three buffer sets: batch b's
    # H2D (copy stream), fused launch (the compute stream, so batches apply
    # in order) and D2H of its results (a second copy stream) overlap the
    # neighbouring batches' stages; every step still moves its own inputs in
    # and its own results out inside the timed region.
    RING = 3
    s_types = [torch.empty(n, dtype=torch.uint8, device="cuda") for _ in range(RING)]
    s_keys = [torch.empty(n, dtype=torch.int64, device="cuda") for _ in range(RING)]
    s_vals = [torch.empty(n, dtype=torch.int64, device="cuda") for _ in range(RING)]
    s_out = [torch.empty((n, 2), dtype=torch.int64, device="cuda") for _ in range(RING)]
    h_outs = [h_out] + [torch.empty((n, 2), dtype=torch.int64).pin_memory()
                        for _ in range(RING - 1)]
    up, down = torch.cuda.Stream(), torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(RING)]
    ev_done = [torch.cuda.Event() for _ in range(RING)]
    ev_out = [torch.cuda.Event() for _ in range(RING)]
    for e in ev_out:
        e.record(down)

    def e2e_step(b):
        r = b % RING
        with torch.cuda.stream(up):
            up.wait_event(ev_out[r])  # the slot's previous results have left
            s_types[r].copy_(h_types[b], non_blocking=True)
            s_keys[r].copy_(h_keys[b], non_blocking=True)
            s_vals[r].copy_(h_vals[b], non_blocking=True)
            ev_in[r].record(up)
        stream.wait_event(ev_in[r])
        fused.execute_fused(s_types[r], s_keys[r], s_vals[r], s_out[r], stream=stream)
        ev_done[r].record(stream)
        with torch.cuda.stream(down):
            down.wait_event(ev_done[r])
            h_outs[r].copy_(s_out[r], non_blocking=True)
            ev_out[r].record(down)

    for b in range(args.warmup):
        e2e_step(b)
    torch.cuda.synchronize()
    ee0, ee1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ee0.record(up)
    for s in range(args.steps):
        e2e_step(args.warmup + s)
    ee1.record(down)
    torch.cuda.synchronize()
    wall_e2e = time.perf_counter() - t0
    barrier(world)
    e2e_ms = max_over_ranks(ee0.elapsed_time(ee1), world)

    # the same pipeline without the table call (each step's results buffer
    # goes back as it is): the rate the host link alone allows
    def copy_step(b):
        r = b % RING
        with torch.cuda.stream(up):
            up.wait_event(ev_out[r])
            s_types[r].copy_(h_types[b], non_blocking=True)
            s_keys[r].copy_(h_keys[b], non_blocking=True)
            s_vals[r].copy_(h_vals[b], non_blocking=True)
            ev_in[r].record(up)
        with torch.cuda.stream(down):
            down.wait_event(ev_in[r])
            h_outs[r].copy_(s_out[r], non_blocking=True)
            ev_out[r].record(down)

    for b in range(args.warmup):
        copy_step(b)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    ee0.record(up)
    for s in range(args.steps):
        copy_step(args.warmup + s)
    ee1.record(down)
    torch.cuda.synchronize()
    barrier(world)
    copy_ms = max_over_ranks(ee0.elapsed_time(ee1), world)

    clk = clocks.stop()
    st |= fused.status()

    ops_rank = n * args.steps
    ops_total = ops_rank * world
    value = ops_total / (fused_ms * 1e-3) / 1e6
    per_batch_value = ops_total / (per_batch_ms * 1e-3) / 1e6
    plain_value = ops_total / (plain_ms * 1e-3) / 1e6
    e2e_value = ops_total / (e2e_ms * 1e-3) / 1e6
    ab = [alg_bytes(batches[args.warmup + s]) for s in range(args.steps)]
    achieved = sum(ab) / (queue_ms * 1e-3) / 1e9  # the timed call
    peak, peak_kind = peaks()
    tuning = fused.tuning()
    overlap = tuning.get("overlap", 0) == 1
    # per-window DRAM bytes of the timed form, from the committed ncu summary
    # of a one-batch capture (not measured in this run)
    traffic_src = "overlap_window_cfg2" if overlap else "fused_map_cfg2"
    traffic = profiled_traffic(traffic_src)
    windows = args.steps * ((n + (1 << 20) - 1) >> 20)  # default window: 2^20 ops
    if overlap:
        form = ("batched call (execute_fused) over the queue of timed batches, one 2^20-op "
                "window per batch: its reads in the lean read kernel on the caller's stream "
                "while its puts are listed, probed, grouped and ordered on a second, "
                "higher-priority stream, then one resolve launch (value); the same call one "
                "batch at a time (per_batch_launch_value); per-op-type calls: a get call and "
                "a put call per batch (plain_value)")
        launches = 5 * windows
    else:
        form = ("fused persistent kernel draining the queue of timed batches in one "
                "launch (value); the same kernel one launch per batch "
                "(per_batch_launch_value); per-op-type launches: a get call and a put "
                "call per batch (plain_value)")
        launches = 1

    line = {
        "metric": METRIC,
        "value": round(value, 2),
        "unit": "Mops/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(fused_ms / args.steps, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u64",
        "data": "synthetic (seeded splitmix64 keys, Zipf 0.99 ranks)",
        "config": {
            "workload": (f"map<u64,u64> 2^{args.buckets_log2} buckets prefilled with "
                         f"2^{args.prefill_log2} keys; batches of 2^{args.batch_log2} ops, "
                         f"{100 - 100 * args.put_frac:.0f}/{100 * args.put_frac:.0f} get/put, "
                         f"Zipf {args.theta} over the prefill keys, gets then puts per batch"),
            "buckets_log2": args.buckets_log2,
            "prefill_log2": args.prefill_log2,
            "batch_ops": n,
            "form": form,
            "lock_mode": args.lock_mode,
            "tuning": tuning,
            "l2": ("no flush: table 2^%d x 480 B = %.1f GB > L2; each step a distinct batch"
                   % (args.buckets_log2, (1 << args.buckets_log2) * 480 / 1e9)),
            "parallelism": f"{world} independent table shard(s), one per GPU",
        },
        "plain_value": round(plain_value, 2),
        "fused_over_plain": round(value / plain_value, 3),
        "per_batch_launch_value": round(per_batch_value, 2),
        "per_batch_launch_over_plain": round(per_batch_value / plain_value, 3),
        "results_identical_fused_vs_plain": identical,
        "device_status": st,
        "e2e": {"value": round(e2e_value, 2), "unit": "Mops/s",
                "h2d_bytes_per_step": int(n * 17), "d2h_bytes_per_step": int(n * 16),
                "wall_s": round(wall_e2e, 4),
                "pipeline": "H2D, the batched call and D2H of consecutive batches on three "
                            "streams, three buffer sets",
                "copy_only_value": round(ops_total / (copy_ms * 1e-3) / 1e6, 2),
                "copy_only": "the same pipeline and bytes without the table call",
                "frac_of_copy_only": round(copy_ms / e2e_ms, 3)},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                     "unit": "GB/s", "frac": round(achieved / peak, 4),
                     "traffic": traffic,
                     "traffic_source": (f"profiles/{traffic_src}.txt: ncu DRAM bytes of one "
                                        "2^20-op batch of this workload (committed capture, "
                                        "not this run)"),
                     "peak_kind": f"{peak_kind} copy bandwidth",
                     "alg_bytes_per_op": round(statistics.mean(ab) / n, 2),
                     "gather_ceiling": {
                         "gets_mops": round(cal_gets / (cal_ms * 1e-3) / 1e6, 1),
                         "batch_floor_us": round(cal_ms * 1e3 / args.steps, 2),
                         "frac": round(cal_ms / fused_ms, 4),
                         "what": ("the accesses of each batch's gets at uniformly random keys "
                                  "of the same 2^%d-bucket table and nothing else (meta sector, "
                                  "then a slot of the same slab; lsb_probe_calibrate); frac = "
                                  "that time / the batch's time" % args.buckets_log2)}},
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args, batches)
        line["cpu_umap"] = cpu_umap(args, batches)
    if rank == 0 and world == 1 and not args.no_side:
        fused.close()
        plain.close()
        del q_types, q_keys, q_vals, q_out, d_types, d_keys, d_vals, out_f, out_g, out_p
        torch.cuda.empty_cache()
        line.update(side_workloads(args, world, rank, local))
    if rank == 0:
        print(json.dumps(line), flush=True)


def side_workloads(args, world, rank, local) -> dict:
    """Compact summaries of the other benchmark configurations, for the
    headline line: the plain method at small size against lslab's own get,
    the uneven-batches stream (fused graph against the per-op-type calls),
    and the serving loop's latency sweep.  Each runs after the timed headline
    region, with its own timing."""
    side = argparse.Namespace(**vars(args))
    side.steps = 5
    out = {}
    ps = run_plain_small(side, world, rank, local)
    out["plain_small"] = {k: ps.get(k) for k in ("ours_mops", "lslab_mops", "ours_over_lslab",
                                                  "results_identical", "hit_fraction")}
    bt = run_batches(side, world, rank, local)
    out["batches"] = {k: bt.get(k) for k in ("fused_mops", "plain_mops", "fused_over_plain",
                                              "plain_issue", "plain_python_mops",
                                              "results_identical", "ops", "batches",
                                              "device_status")}
    # the serving loop at two wave limits: 2^16 ops (throughput) and 2^14
    # (latency: smaller waves, lower peak)
    for key, wave in (("serving", 1 << 16), ("serving_wave_2e14", 1 << 14)):
        side.wave_ops = wave
        sv = run_serving(side, world, rank, local)
        at70 = [p for p in sv["sweep"] if abs(p["load"] - 0.7) < 1e-9]
        out[key] = {
            "peak_mops": sv["peak_mops"], "wave_ops": sv["wave_ops"],
            "peak_wave_split": sv["peak_wave_split"],
            "at_70pct": at70[0] if at70 else None,
            "p99_us_by_load": {str(p["load"]): p["p99_us"] for p in sv["sweep"]},
            "loop_state": sv["loop"]["state"], "device_status": sv["device_status"],
        }
    return out


def cpu_baseline(args, batches):
    """The oracle (plain-C restatement of the reference's slab list) replaying
    a bounded sample of the same workload on the host cores, bucket-sharded
    over threads (results identical to the sequential replay)."""
    from oracle import OracleMap
    threads = max(1, min(32, os.cpu_count() or 1))
    pk, pv = prefill_arrays(args, 0)
    o = OracleMap(args.buckets_log2, 1 << 16)
    chunk = 1 << 22
    put_t = np.ones(chunk, np.uint8)
    for off in range(0, len(pk), chunk):
        k = pk[off:off + chunk]
        o.mixed(put_t[:len(k)], k, pv[off:off + chunk], threads=threads)
    nb = min(args.cpu_batches, len(batches))
    t0 = time.perf_counter()
    ops = 0
    reps = 0
    while True:  # cycle the sample batches for at least cpu_seconds of wall time
        for b in batches[:nb]:
            o.mixed(b.types, b.keys, b.vals, threads=threads)
            ops += len(b.keys)
        reps += 1
        if time.perf_counter() - t0 >= args.cpu_seconds:
            break
    dt = time.perf_counter() - t0
    return {"value": round(ops / dt / 1e6, 2), "unit": "Mops/s", "cores": threads,
            "kind": "port",
            "sample": f"{nb} batches of {len(batches[0].keys)} ops replayed {reps}x "
                      f"({ops} ops) on the full-size table (2^{args.buckets_log2} buckets, "
                      f"2^{args.prefill_log2} prefill): {dt:.2f} s wall on {threads} threads"}


def cpu_umap(args, batches):
    """std::unordered_map<uint64_t, uint64_t> host replay of a bounded sample of
    the same workload (oracle/umap_replay.cpp): the prefill keys in per-core
    shard maps (filled in parallel, untimed), then the sample batches replayed
    in op-index order by one thread, and by one thread per shard."""
    from oracle import UmapReplay
    shards = max(1, min(32, os.cpu_count() or 1))
    pk, pv = prefill_arrays(args, 0)
    u = UmapReplay(pk, pv, shards=shards)
    nb = min(args.cpu_batches, len(batches))
    out = {}
    for threads in (1, shards):
        ops, dt, reps = 0, 0.0, 0
        while dt < args.cpu_seconds / 2:
            for b in batches[:nb]:
                t, _ = u.replay(b.types, b.keys, b.vals, threads=threads, want_results=False)
                dt += t
                ops += len(b.keys)
            reps += 1
        out[threads] = (ops / dt / 1e6, ops, dt, reps)
    u.close()
    v1, ops1, dt1, reps1 = out[1]
    vs, opss, dts, repss = out[shards]
    return {"value": round(v1, 2), "unit": "Mops/s", "cores": 1,
            "kind": "std::unordered_map replay",
            "sample": f"{nb} batches of {len(batches[0].keys)} ops replayed {reps1}x ({ops1} ops, "
                      f"{dt1:.2f} s, steady_clock) after a 2^{args.prefill_log2}-key prefill",
            "sharded_value": round(vs, 2), "sharded_cores": shards,
            "sharded_sample": f"the same batches {repss}x ({opss} ops, {dts:.2f} s), one thread "
                              f"per hash shard, each in op-index order"}


# ------------------------------------------------------------ reference arm
def run_reference(args, world, rank, local):
    import torch
    import oracle
    from oracle import RefMap, ref_map_pool_bound

    if rank != 0:
        return  # rank 0 alone runs the reference arm
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/liblslab_ref.so not built"}))
        return
    stream = torch.cuda.current_stream()
    n = 1 << args.batch_log2
    nb = args.warmup + args.steps
    batches = make_batches(args, 0, nb)
    pk, pv = prefill_arrays(args, 0)
    inserts = np.concatenate([pk] + [b.keys[b.types == 1] for b in batches])
    pool = ref_map_pool_bound(args.buckets_log2, inserts)
    del inserts
    m = RefMap(args.buckets_log2, pool)
    for off in range(0, len(pk), 1 << 22):
        k = dev_u64(torch, pk[off:off + (1 << 22)])
        v = dev_u64(torch, pv[off:off + (1 << 22)])
        old = torch.empty_like(k)
        m.put(k, v, old, stream.cuda_stream)
    torch.cuda.synchronize()
    d_keys = [dev_u64(torch, b.keys) for b in batches]
    d_vals = [dev_u64(torch, b.vals) for b in batches]
    n_get = [int(np.sum(b.types == 0)) for b in batches]
    out_g = torch.empty((n, 2), dtype=torch.int64, device="cuda")
    out_p = torch.empty(n, dtype=torch.int64, device="cuda")

    def step(b, keys, vals):
        g = n_get[b]
        m.get(keys[:g], out_g[:g], stream.cuda_stream)
        m.put(keys[g:], vals[g:], out_p[: n - g], stream.cuda_stream)

    clocks = Clocks(local)
    for b in range(args.warmup):
        step(b, d_keys[b], d_vals[b])
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for s in range(args.steps):
        b = args.warmup + s
        step(b, d_keys[b], d_vals[b])
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)

    # e2e: host buffers, copies inside the timed region, pipelined exactly as
    # in our arm (copy-in stream, compute stream, copy-out stream, a ring of
    # three buffer sets)
    RING = 3
    h_keys = [torch.from_numpy(b.keys.view(np.int64)).pin_memory() for b in batches]
    h_vals = [torch.from_numpy(b.vals.view(np.int64)).pin_memory() for b in batches]
    h_out = [torch.empty((n, 2), dtype=torch.int64).pin_memory() for _ in range(RING)]
    h_old = [torch.empty(n, dtype=torch.int64).pin_memory() for _ in range(RING)]
    s_keys = [torch.empty(n, dtype=torch.int64, device="cuda") for _ in range(RING)]
    s_vals = [torch.empty(n, dtype=torch.int64, device="cuda") for _ in range(RING)]
    r_g = [torch.empty((n, 2), dtype=torch.int64, device="cuda") for _ in range(RING)]
    r_p = [torch.empty(n, dtype=torch.int64, device="cuda") for _ in range(RING)]
    up, down = torch.cuda.Stream(), torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(RING)]
    ev_done = [torch.cuda.Event() for _ in range(RING)]
    ev_out = [torch.cuda.Event() for _ in range(RING)]
    for e in ev_out:
        e.record(down)
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(up)
    for s in range(args.steps):
        b = args.warmup + s
        r = b % RING
        g = n_get[b]
        with torch.cuda.stream(up):
            up.wait_event(ev_out[r])
            s_keys[r].copy_(h_keys[b], non_blocking=True)
            s_vals[r].copy_(h_vals[b], non_blocking=True)
            ev_in[r].record(up)
        stream.wait_event(ev_in[r])
        m.get(s_keys[r][:g], r_g[r][:g], stream.cuda_stream)
        m.put(s_keys[r][g:], s_vals[r][g:], r_p[r][: n - g], stream.cuda_stream)
        ev_done[r].record(stream)
        with torch.cuda.stream(down):
            down.wait_event(ev_done[r])
            h_out[r][:g].copy_(r_g[r][:g], non_blocking=True)
            h_old[r][: n - g].copy_(r_p[r][: n - g], non_blocking=True)
            ev_out[r].record(down)
    e3.record(down)
    torch.cuda.synchronize()
    e2e_ms = e2.elapsed_time(e3)
    clk = clocks.stop()
    value = n * args.steps / (ms * 1e-3) / 1e6
    e2e_value = n * args.steps / (e2e_ms * 1e-3) / 1e6
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": round(value, 2),
        "unit": "Mops/s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms / args.steps, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u64",
        "data": "synthetic (seeded splitmix64 keys, Zipf 0.99 ranks)",
        "config": {
            "workload": (f"map<u64,u64> 2^{args.buckets_log2} buckets prefilled with "
                         f"2^{args.prefill_log2} keys; batches of 2^{args.batch_log2} ops, "
                         f"{100 - 100 * args.put_frac:.0f}/{100 * args.put_frac:.0f} get/put, "
                         f"Zipf {args.theta} over the prefill keys, gets then puts per batch"),
            "form": "lslab map::get<256> then map::put<256> per batch (its only batched form)",
        },
        "reference": ("depaulmillz/lslab's own map kernels built for sm_100a from its headers; "
                      "the reference has no CPU implementation of this path"),
        "cpu_baseline": {"value": round(value, 2), "unit": "Mops/s", "cores": 0,
                         "kind": "reference",
                         "sample": (f"{args.steps} batches of {n} ops on the GPU (the reference "
                                    "is GPU-only; no host cores do the work)")},
        "e2e": {"value": round(e2e_value, 2), "unit": "Mops/s", "h2d_bytes_per_step": n * 16,
                "d2h_bytes_per_step": int(statistics.mean(16 * g + 8 * (n - g) for g in n_get)),
                "pipeline": "H2D, get+put launches and D2H of consecutive batches on three "
                            "streams, three buffer sets"},
        "pool_slabs_used": m.pool_used(),
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def run_batches(args, world, rank, local):
    """4096 mixed get/put/remove batches (lognormal sizes, median 512, sigma
    1.5, clipped to [1, 2^18]; 80/15/5; Zipf 0.99 over 2^27 keys) on a map with
    2^24 buckets prefilled with the 2^26 most popular keys.  Fused: the whole
    batch stream as one autotuned, CUDA-graph-captured persistent launch.
    Plain: per batch, one call per op type (get, put, remove), as the
    reference's API issues them.  Results and final contents checked equal."""
    import torch
    import lslab_b200 as L
    from lslab_b200 import workload as W
    from lslab_b200.shard import rank_seed

    seed = rank_seed(args.seed, rank)
    log2, items, pre = 24, 1 << 27, 1 << 26
    sizes = W.lognormal_sizes(seed, args.nbatches, 512, 1.5, 1, 1 << 18)
    parts = [W.map_zipf_batch(seed, b, int(n), items, 0.99, (0.8, 0.15, 0.05))
             for b, n in enumerate(sizes)]
    types = np.concatenate([p.types for p in parts])
    keys = np.concatenate([p.keys for p in parts])
    vals = np.concatenate([p.vals for p in parts])
    n = len(keys)
    pk = W.key_of_rank(seed, np.arange(pre))
    fused = L.Map(log2, 1 << 22)
    plain = L.Map(log2, 1 << 22)
    for off in range(0, pre, 1 << 24):
        k = dev_u64(torch, pk[off:off + (1 << 24)])
        fused.put(k, k)
        plain.put(k, k)
        del k
    d_types = torch.from_numpy(types).cuda()
    d_keys, d_vals = dev_u64(torch, keys), dev_u64(torch, vals)
    out_f = torch.empty((n, 2), dtype=torch.int64, device="cuda")
    # autotune on a sample (the first 256 batches); the plain table gets the
    # sample once as well, so both tables stay identical
    ns = int(sum(sizes[:256]))
    if args.no_autotune:
        apply_tuning(args, fused)
        fused.execute_fused(d_types[:ns], d_keys[:ns], d_vals[:ns], out_f[:ns])
        tuned = fused.tuning()
    else:
        tuned = fused.autotune(d_types[:ns], d_keys[:ns], d_vals[:ns], out_f[:ns])
    plain.execute(d_types[:ns], d_keys[:ns], d_vals[:ns], out_f[:ns])
    graph = fused.capture_fused(d_types, d_keys, d_vals, out_f)
    offs = np.concatenate([[0], np.cumsum(sizes)])
    cnt = [(int(np.sum(p.types == 0)), int(np.sum(p.types == 1))) for p in parts]
    d_out_g = torch.empty((n, 2), dtype=torch.int64, device="cuda")
    d_out_p = torch.empty(n, dtype=torch.int64, device="cuda")

    d_out_g2 = torch.empty((n, 2), dtype=torch.int64, device="cuda")
    d_out_p2 = torch.empty(n, dtype=torch.int64, device="cuda")

    def plain_pass(st=None, out_g=d_out_g, out_p=d_out_p):
        for b, (g, p) in enumerate(cnt):
            o = int(offs[b])
            r = int(sizes[b]) - g - p
            if g:
                plain.get(d_keys[o:o + g], out_g[o:o + g], stream=st)
            if p:
                plain.put(d_keys[o + g:o + g + p], d_vals[o + g:o + g + p], out_p[o + g:o + g + p],
                          stream=st)
            if r:
                plain.remove(d_keys[o + g + p:o + g + p + r], out_g[o + g + p:o + g + p + r],
                             stream=st)

    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    reps = max(1, args.steps)
    f_ms, p_ms, pg_ms, identical = [], [], [], True
    cap = torch.cuda.Stream()
    for rep in range(reps):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(6)]
        e[0].record(stream)
        graph.launch()
        e[1].record(stream)
        e[2].record(stream)
        plain_pass()  # issued from Python: one ctypes call per op type per batch
        e[3].record(stream)
        torch.cuda.synchronize()
        f_ms.append(e[0].elapsed_time(e[1]))
        p_ms.append(e[2].elapsed_time(e[3]))
        # the same per-op-type calls captured into one CUDA graph, so the GPU
        # runs them without host issue gaps (captured afresh for each replay:
        # a replay runs every captured window once, so no window epoch
        # repeats).  The plain table takes the stream once more; a key's final
        # state is its last mutation in the stream, so the contents still
        # equal the fused table's; results go to separate buffers.
        pg = torch.cuda.CUDAGraph()
        with torch.cuda.graph(pg, stream=cap):
            plain_pass(cap, d_out_g2, d_out_p2)
        e[4].record(stream)
        pg.replay()
        e[5].record(stream)
        torch.cuda.synchronize()
        pg_ms.append(e[4].elapsed_time(e[5]))
        del pg
        if rep == 0:
            # fused results vs the per-type calls of the same batches
            isput = torch.from_numpy(types == 1).cuda()
            got_f = out_f.clone()
            want = d_out_g.clone()
            want[isput, 0] = -1  # put results compared on the value only
            got_f[isput, 0] = -1
            want[isput, 1] = d_out_p[isput]
            identical = bool(torch.equal(got_f, want))
    kf, vf = fused.dump()
    kp, vp = plain.dump()
    identical = identical and np.array_equal(kf, kp) and np.array_equal(vf, vp)
    graph.close()
    fm, pm, pgm = statistics.median(f_ms), statistics.median(p_ms), statistics.median(pg_ms)
    line = {
        "workload": "batches",
        "description": (f"{args.nbatches} mixed batches (lognormal median 512, sigma 1.5), "
                        f"80/15/5 get/put/remove, Zipf 0.99 over 2^27 keys, map 2^24 "
                        f"buckets prefilled with 2^26 keys"),
        "ops": n, "batches": args.nbatches, "reps": reps,
        "fused_mops": round(n / (fm * 1e-3) / 1e6, 1),
        "plain_mops": round(n / (pgm * 1e-3) / 1e6, 1),
        "fused_over_plain": round(pgm / fm, 2),
        "plain_issue": "per-op-type calls captured in one CUDA graph",
        "plain_python_mops": round(n / (pm * 1e-3) / 1e6, 1),
        "fused_ms": [round(x, 3) for x in f_ms], "plain_ms": [round(x, 3) for x in pg_ms],
        "plain_python_ms": [round(x, 2) for x in p_ms],
        "results_identical": identical, "tuning": tuned,
        "plain_calls_per_pass": int(sum((g > 0) + (p > 0) + (int(sizes[b]) - g - p > 0)
                                        for b, (g, p) in enumerate(cnt))),
        "fused_launches_per_pass": 1,
        "device_status": fused.status() | plain.status(),
    }
    fused.close()
    plain.close()
    return line


def run_serving(args, world, rank, local):
    """Serving (map 2^25 buckets, slab pool capped at 24 GB): requests of
    uniform [1, 4096] ops, 50/50 get/put, Zipf 0.99 over 2^28 keys, fed by the
    open-loop generator (lsb_serve_run_load) from a pool of 4096 requests.
    Peak = throughput with the queue never empty; then Poisson arrivals at
    fractions of that peak, each point reporting achieved Mops/s and the
    p50/p99/p999 latency from scheduled arrival to observed completion."""
    import lslab_b200 as L
    from lslab_b200 import workload as W
    from lslab_b200.shard import rank_seed

    seed = rank_seed(args.seed, rank)
    pool_slabs = 24_000_000_000 // 480
    m = L.Map(25, pool_slabs)
    apply_tuning(args, m)  # the loop's launch shape (block threads, lookahead)
    srv = L.Server(m, max_wave_ops=args.wave_ops, ring_requests=16384, arena_ops=1 << 22)
    off, n, t, k, v = W.serving_pool(seed, 4096)
    mean_n = float(n.mean())
    rng = np.random.default_rng(seed)
    srv.start()

    def run(nreq, arrival):
        idx = rng.integers(0, len(n), size=nreq).astype(np.uint32)
        q0 = srv.query()
        lat, wall, _ = srv.run_load(arrival, idx, off, n, t, k, v)
        q1 = srv.query()
        ops = int(n[idx].astype(np.uint64).sum())
        return lat, wall, ops, wave_split(q0, q1)

    def wave_split(q0, q1):
        # the loop's own step times over the waves of one run (lsb_serve_query)
        w = max(1, q1["waves"] - q0["waves"])
        return {"waves": q1["waves"] - q0["waves"],
                "ops_per_wave": round((q1["ops"] - q0["ops"]) / w, 1),
                **{f"{key}_us_per_wave": round((q1[f"{key}_ns"] - q0[f"{key}_ns"]) / w / 1e3, 2)
                   for key in ("gather", "engine", "tail")},
                "wait_us_total": round((q1["wait_ns"] - q0["wait_ns"]) / 1e3, 1)}

    run(512, np.zeros(512, np.uint64))  # warm-up
    peak_req = 8192
    _, wall, ops, peak_split = run(peak_req, np.zeros(peak_req, np.uint64))
    peak = ops / (wall * 1e-9)
    sweep = []
    for f in [float(x) for x in args.serve_loads.split(",")]:
        lam = f * peak / mean_n  # requests per second
        nreq = max(256, int(lam * args.serve_seconds))
        arrival = np.cumsum(rng.exponential(1e9 / lam, size=nreq)).astype(np.uint64)
        lat, wall, ops, split = run(nreq, arrival)
        us = lat / 1e3
        sweep.append({"load": f, "offered_mops": round(f * peak / 1e6, 1),
                      "achieved_mops": round(ops / (wall * 1e-9) / 1e6, 1), "requests": nreq,
                      "p50_us": round(float(np.percentile(us, 50)), 1),
                      "p99_us": round(float(np.percentile(us, 99)), 1),
                      "p999_us": round(float(np.percentile(us, 99.9)), 1),
                      "wave_split": split})
    stats = srv.stop()
    srv.close()
    at70 = [p for p in sweep if abs(p["load"] - 0.7) < 1e-9]
    line = {
        "workload": "serving",
        "description": ("map 2^25 buckets, slab pool capped at 24 GB; requests uniform [1, 4096] "
                        "ops, 50/50 get/put, Zipf 0.99 over 2^28 keys; open-loop Poisson "
                        "arrivals; latency = scheduled arrival to observed completion"),
        "wave_ops": args.wave_ops, "peak_mops": round(peak / 1e6, 1), "peak_wave_split": peak_split,
        "p99_us_at_70pct": at70[0]["p99_us"] if at70 else None,
        "sweep": sweep, "loop": stats, "device_status": m.status(),
        "pool_slabs_used": m.pool_usage()[0],
    }
    m.close()
    return line


def _perm32(torch, idx):
    """Distinct u32 keys on the device: a bijective 32-bit mix of `idx`
    (odd multiplies and xor-shifts modulo 2^32), as int32 tensors."""
    m = 0xFFFFFFFF
    x = idx.to(torch.int64) & m
    x = ((x ^ (x >> 16)) * 0x7FEB352D) & m
    x = ((x ^ (x >> 15)) * 0x846CA68B) & m
    x = x ^ (x >> 16)
    return (x - ((x >> 31) << 32)).to(torch.int32)  # two's-complement view


def run_sets(args, world, rank, local):
    """Set load-factor sweep: set<u32> with 2^18 buckets (42 MB of head slabs,
    L2-resident) and 2^24 buckets (2.7 GB of heads plus the chains the load
    needs, HBM-resident), prefilled to 0.25 .. 4 keys per head-slab slot;
    batches of 2^18 ops, 40% insert / 50% contains / 10% remove over a
    universe of the prefill keys and as many absent keys (uniform).  Fused:
    one execute_fused per batch; plain: per batch the insert, contains and
    remove calls of its type-sorted parts; lslab: the same calls through the
    reference's own kernels.  Checks: fused and plain give identical results
    for every batch; lslab's contains results equal ours, its removes report
    as many hits, and after the run a sample of 2^20 universe keys is
    contained in lslab's table exactly where it is in ours."""
    import torch
    import lslab_b200 as L
    import oracle
    from oracle import RefSet
    from lslab_b200.shard import rank_seed

    seed = rank_seed(args.seed, rank)
    gen = torch.Generator(device="cuda")
    n = 1 << 18
    nb = args.warmup + args.steps
    have_ref = oracle.ref_available()
    points = []
    forms = [f for f in args.set_forms.split(",") if f]
    for log2 in [int(x) for x in args.set_log2.split(",")]:
        for lf in [float(x) for x in args.set_lf.split(",")]:
            nk = int(lf * (1 << log2) * 28)
            pool = max(4096, int(nk / 28 * 1.5) + (1 << log2) // 4)
            gen.manual_seed(seed + log2 * 100 + int(lf * 8))
            batches = []
            for _ in range(nb):
                u = torch.rand(n, device="cuda", generator=gen)
                ty = torch.where(u < 0.4, 1, torch.where(u < 0.9, 0, 2)).to(torch.uint8)
                ty, _ = torch.sort(ty)  # contains, insert, remove: type-sorted parts
                idx = torch.randint(0, 2 * nk, (n,), device="cuda", generator=gen)
                batches.append((ty, _perm32(torch, idx)))
            cnt = [(int((b[0] == 0).sum()), int((b[0] == 1).sum())) for b in batches]
            sample = _perm32(torch, torch.randint(0, 2 * nk, (1 << 20,), device="cuda",
                                                  generator=gen))
            res, outs, held = {}, {}, {}
            for form in forms:
                if form == "lslab":
                    if not have_ref:
                        continue
                    # lslab's identity hash (hash.h:12-14): a bucket's slabs
                    # never exceed ceil(its inserts / 31)
                    per = torch.zeros(1 << log2, dtype=torch.int64, device="cuda")
                    mask = (1 << log2) - 1
                    for off in range(0, nk, 1 << 24):
                        k = _perm32(torch, torch.arange(off, min(nk, off + (1 << 24)),
                                                        device="cuda"))
                        per += torch.bincount(k.to(torch.int64) & mask, minlength=1 << log2)
                    for (ty, k), (c, ins) in zip(batches, cnt):
                        per += torch.bincount(k[c:c + ins].to(torch.int64) & mask,
                                              minlength=1 << log2)
                    bound = int(torch.clamp((per + 30) // 31 - 1, min=0).sum()) + 64
                    del per
                    st = RefSet(log2, bound)
                    tmp = torch.empty(1 << 24, dtype=torch.bool, device="cuda")
                else:
                    st = L.Set(log2, pool)
                for off in range(0, nk, 1 << 24):
                    k = _perm32(torch, torch.arange(off, min(nk, off + (1 << 24)), device="cuda"))
                    if form == "lslab":
                        st.insert(k, tmp[:k.numel()])
                    else:
                        st.insert(k)
                    del k
                torch.cuda.synchronize()
                out = torch.empty((nb, n), dtype=torch.bool, device="cuda")

                def step(i):
                    ty, k = batches[i]
                    o = out[i]
                    if form == "fused":
                        st.execute_fused(ty, k, o)
                        return
                    c, ins = cnt[i]
                    if c:
                        st.contains(k[:c], o[:c])
                    if ins:
                        st.insert(k[c:c + ins], o[c:c + ins])
                    if n - c - ins:
                        st.remove(k[c + ins:], o[c + ins:])
                for i in range(args.warmup):
                    step(i)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record()
                for i in range(args.warmup, nb):
                    step(i)
                e1.record()
                torch.cuda.synchronize()
                res[form] = round(args.steps * n / (e0.elapsed_time(e1) * 1e-3) / 1e6, 1)
                held_out = torch.empty(sample.numel(), dtype=torch.bool, device="cuda")
                st.contains(sample, held_out)
                torch.cuda.synchronize()
                held[form] = held_out
                outs[form] = out
                if form != "lslab":
                    res["status"] = res.get("status", 0) | st.status()
                st.close()
                del st
            both = "fused" in outs and "plain" in outs
            ident = bool(torch.equal(outs["fused"], outs["plain"])) if both else None
            vs_ref = None
            if "lslab" in outs and "fused" in outs:
                a, r = outs["fused"], outs["lslab"]
                same_contains = all(torch.equal(a[i, :c], r[i, :c]) for i, (c, _) in enumerate(cnt))
                same_removes = all(int(a[i, c + ins:].sum()) == int(r[i, c + ins:].sum())
                                   for i, (c, ins) in enumerate(cnt))
                vs_ref = bool(same_contains and same_removes
                              and torch.equal(held["fused"], held["lslab"]))
            points.append({"buckets_log2": log2, "keys_per_slot": lf, "keys": nk,
                           "head_mb": round((1 << log2) * 160 / 1e6, 1),
                           "fused_mops": res.get("fused"), "plain_mops": res.get("plain"),
                           "lslab_mops": res.get("lslab"),
                           "results_identical_fused_plain": (ident and bool(torch.equal(
                               held["fused"], held["plain"]))) if both else None,
                           "results_match_lslab": vs_ref,
                           "device_status": res.get("status", 0)})
            del outs, held, batches, sample
            torch.cuda.empty_cache()
    if rank == 0:
        print(json.dumps({"workload": "sets", "description": run_sets.__doc__.split(".")[0],
                          "batch_ops": n, "steps": args.steps, "points": points}), flush=True)
    return points


def run_probes(args, world, rank, local):
    """Probe comparison on read-only batches: the thread-per-op tag probe
    (default: a 32-B meta sector, then the candidate slot) against the
    warp-cooperative slab probe of the reference's design (tuning
    warp_probe=1: a warp serves its lanes' distinct keys one at a time,
    lanes reading a slab's slots together).  The headline map (2^22 buckets,
    2^26 keys, the gets of 2^20-op 95/5 Zipf batches) and sets at 1 key per
    head-slab slot (2^18 and 2^22 buckets, 2^18-op contains batches, half
    present); same inputs and results checked identical."""
    import torch
    import lslab_b200 as L
    from lslab_b200 import workload as W
    from lslab_b200.shard import rank_seed

    seed = rank_seed(args.seed, rank)
    reps = max(3, args.steps)

    def timed(fn, inputs, out):
        for x in inputs[:2]:
            fn(x, out)
        torch.cuda.synchronize()
        ts = []
        for x in inputs[2:2 + reps]:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn(x, out)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    points = []
    pk, pv = prefill_arrays(args, rank)
    m = L.Map(args.buckets_log2, max(1 << (args.buckets_log2 - 2), 4096))
    for off in range(0, len(pk), 1 << 24):
        m.put(dev_u64(torch, pk[off:off + (1 << 24)]), dev_u64(torch, pv[off:off + (1 << 24)]))
    batches = make_batches(args, rank, reps + 2)
    gets = [dev_u64(torch, b.keys[b.types == 0]) for b in batches]
    n = max(int(g.numel()) for g in gets)
    res = {}
    for wp in (0, 1):
        m.set_tuning(warp_probe=wp)
        out = torch.empty((n, 2), dtype=torch.int64, device="cuda")
        ms = timed(lambda k, o: m.get(k, o[:k.numel()]), gets, out)
        res[wp] = (ms, out[:gets[-1].numel()].clone())
    same = bool(torch.equal(res[0][1], res[1][1]))
    points.append({"table": f"map 2^{args.buckets_log2} buckets, 2^{args.prefill_log2} keys",
                   "ops": int(gets[2].numel()), "tag_probe_us": round(res[0][0] * 1e3, 1),
                   "warp_probe_us": round(res[1][0] * 1e3, 1),
                   "tag_over_warp": round(res[1][0] / res[0][0], 2), "results_identical": same})
    m.close()
    del gets
    for log2 in (18, 22):
        nk = (1 << log2) * 28
        st = L.Set(log2, nk // 28 + 4096)
        for off in range(0, nk, 1 << 24):
            st.insert(_perm32(torch, torch.arange(off, min(nk, off + (1 << 24)), device="cuda")))
        gen = torch.Generator(device="cuda")
        gen.manual_seed(seed + log2)
        qs = [_perm32(torch, torch.randint(0, 2 * nk, (1 << 18,), device="cuda", generator=gen))
              for _ in range(reps + 2)]
        r = {}
        for wp in (0, 1):
            st.set_tuning(warp_probe=wp)
            out = torch.empty(1 << 18, dtype=torch.bool, device="cuda")
            ms = timed(lambda k, o: st.contains(k, o), qs, out)
            r[wp] = (ms, out.clone())
        points.append({"table": f"set 2^{log2} buckets, 1 key per head slot", "ops": 1 << 18,
                       "tag_probe_us": round(r[0][0] * 1e3, 1),
                       "warp_probe_us": round(r[1][0] * 1e3, 1),
                       "tag_over_warp": round(r[1][0] / r[0][0], 2),
                       "results_identical": bool(torch.equal(r[0][1], r[1][1]))})
        st.close()
    return {"workload": "probes", "description": run_probes.__doc__.split(":")[0],
            "reps": reps, "points": points}


def run_locks(args, world, rank, local):
    """Bucket-lock comparison on the map (writer lock = the reference's
    warp_mutex role; lock-free = CAS on slab tag words; rw = reader-writer
    locks on the read path too): 2^20-op batches, Zipf 0.99 over 2^26 keys on
    2^22 buckets prefilled with 2^26 keys, 95/5 and 50/50 get/put, fused and
    per-op-type forms.  Results are identical across modes (tests)."""
    import torch
    import lslab_b200 as L

    n = 1 << args.batch_log2
    nb = args.warmup + args.steps
    pk, pv = prefill_arrays(args, rank)
    pool = max(1 << (args.buckets_log2 - 2), 4096)
    rows = []
    for put_frac in (0.05, 0.5):
        args.put_frac = put_frac
        batches = make_batches(args, rank, nb)
        dT = [torch.from_numpy(b.types).cuda() for b in batches]
        dK = [dev_u64(torch, b.keys) for b in batches]
        dV = [dev_u64(torch, b.vals) for b in batches]
        ng = [int(np.sum(b.types == 0)) for b in batches]
        out = torch.empty((n, 2), dtype=torch.int64, device="cuda")
        old = torch.empty(n, dtype=torch.int64, device="cuda")
        for mode in ("writer", "free", "rw"):
            m = L.Map(args.buckets_log2, pool, lock_mode=mode)
            for off in range(0, len(pk), 1 << 24):
                k = dev_u64(torch, pk[off:off + (1 << 24)])
                v = dev_u64(torch, pv[off:off + (1 << 24)])
                m.put(k, v)
                del k, v
            row = {"put_frac": put_frac, "lock_mode": mode}
            for form in ("fused", "plain"):
                def step(i):
                    if form == "fused":
                        m.execute_fused(dT[i], dK[i], dV[i], out)
                    else:
                        g = ng[i]
                        m.get(dK[i][:g], out[:g])
                        m.put(dK[i][g:], dV[i][g:], old[g:])
                for i in range(args.warmup):
                    step(i)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record()
                for i in range(args.warmup, nb):
                    step(i)
                e1.record()
                torch.cuda.synchronize()
                row[form + "_mops"] = round(args.steps * n / (e0.elapsed_time(e1) * 1e-3) / 1e6, 1)
            row["device_status"] = m.status()
            m.close()
            rows.append(row)
    if rank == 0:
        print(json.dumps({"workload": "locks", "description": run_locks.__doc__.split(".")[0],
                          "rows": rows}), flush=True)


def run_plain_small(args, world, rank, local):
    """Plain method, small size: map with 2^16 buckets, 2^20 distinct
    splitmix64 keys inserted (value = key ^ 0x9E3779B97F4A7C15), then 2^20
    gets (half present keys, half keys of a disjoint stream) in batches of
    2^16, one get call per batch; this library's lsb_map_get against lslab's
    own map::get (built for sm_100a) on the same keys, results compared."""
    import torch
    import lslab_b200 as L
    import oracle
    from oracle import RefMap, ref_map_pool_bound
    from lslab_b200 import workload as W
    from lslab_b200.shard import rank_seed

    if rank != 0:
        return
    seed = rank_seed(args.seed, rank)
    nk, bn = 1 << 20, 1 << 16
    pk = W.prefill_keys(seed, nk)
    pv = W.prefill_values(pk)
    rng = np.random.default_rng(seed)
    present = pk[rng.integers(0, nk, size=nk // 2)]
    absent = W.absent_keys(seed, nk // 2 + 64, pk)[: nk // 2]
    q = np.concatenate([present, absent])
    q = q[rng.permutation(len(q))]
    dq = dev_u64(torch, q)
    reps = max(1, args.steps)

    def timed(get, out):
        for b in range(0, nk, bn):  # warm-up pass
            get(dq[b:b + bn], out[b:b + bn])
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            for b in range(0, nk, bn):
                get(dq[b:b + bn], out[b:b + bn])
        e1.record()
        torch.cuda.synchronize()
        return nk * reps / (e0.elapsed_time(e1) * 1e-3) / 1e6

    res = {}
    m = L.Map(16, max(4096, nk // 28 * 2))
    m.put(dev_u64(torch, pk), dev_u64(torch, pv))
    out_m = torch.empty((nk, 2), dtype=torch.int64, device="cuda")
    res["ours_mops"] = round(timed(lambda k, o: m.get(k, o), out_m), 1)
    status = m.status()
    if oracle.ref_available():
        r = RefMap(16, ref_map_pool_bound(16, pk))
        old = torch.empty(nk, dtype=torch.int64, device="cuda")
        r.put(dev_u64(torch, pk), dev_u64(torch, pv), old)
        out_r = torch.empty((nk, 2), dtype=torch.int64, device="cuda")
        res["lslab_mops"] = round(timed(lambda k, o: r.get(k, o), out_r), 1)
        a, b = out_m.cpu().numpy(), out_r.cpu().numpy()
        found_m = (a[:, 0].view(np.uint64) & np.uint64(0xFF)) != 0
        found_r = (b[:, 0].view(np.uint64) & np.uint64(0xFF)) != 0
        res["results_identical"] = bool(np.array_equal(found_m, found_r) and np.array_equal(
            a[:, 1][found_m], b[:, 1][found_r]))
        res["ours_over_lslab"] = round(res["ours_mops"] / res["lslab_mops"], 2)
        r.close()
    hits = int(((out_m[:, 0] & 0xFF) != 0).sum())
    m.close()
    return {"workload": "plain-small", "description": run_plain_small.__doc__.split(";")[0],
            "gets": nk, "batch_ops": bn, "reps": reps, "hit_fraction": hits / nk,
            **res, "device_status": status}


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank, local)
    elif args.workload == "batches":
        line = run_batches(args, world, rank, local)
        if rank == 0:
            print(json.dumps(line), flush=True)
    elif args.workload == "serving":
        line = run_serving(args, world, rank, local)
        if rank == 0:
            print(json.dumps(line), flush=True)
    elif args.workload == "sets":
        run_sets(args, world, rank, local)
    elif args.workload == "locks":
        run_locks(args, world, rank, local)
    elif args.workload == "probes":
        line = run_probes(args, world, rank, local)
        if rank == 0:
            print(json.dumps(line), flush=True)
    elif args.workload == "plain-small":
        line = run_plain_small(args, world, rank, local)
        if rank == 0:
            print(json.dumps(line), flush=True)
    else:
        run_ours(args, world, rank, local)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
