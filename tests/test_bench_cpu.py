"""CPU checks of bench.py's host-side pieces: the argument defaults the
timing rules need, the algorithmic byte count of the headline mix, and the
two CPU baselines (the oracle replay and the std::unordered_map replay) at a
small size, with the keys their JSON objects carry."""
from __future__ import annotations

import sys

import numpy as np
import pytest

import bench as B


def _args(*extra):
    argv = sys.argv
    try:
        sys.argv = ["bench.py", "--buckets-log2", "10", "--prefill-log2", "14", "--batch-log2", "12",
                    "--cpu-seconds", "0.2", "--cpu-batches", "2", *extra]
        return B.parse()
    finally:
        sys.argv = argv


def test_defaults_follow_the_timing_rules():
    argv = sys.argv
    try:
        sys.argv = ["bench.py"]
        a = B.parse()
    finally:
        sys.argv = argv
    assert a.gpus == 1 and a.warmup >= 3 and a.steps >= 1
    assert a.workload == "zipf9505" and a.impl == "ours"
    assert (a.buckets_log2, a.prefill_log2, a.batch_log2) == (22, 26, 20)


def test_headline_mix_bytes_per_op():
    a = _args()
    (b,) = B.make_batches(a, 0, 1)
    got = B.alg_bytes(b) / len(b.keys)
    nput = float(np.mean(b.types == 1))
    assert got == pytest.approx((1 - nput) * B.BYTES_GET + nput * B.BYTES_PUT)
    assert got == pytest.approx(89.6, abs=0.5)  # 95/5: 0.95 x 88 + 0.05 x 120


@pytest.mark.parametrize("which", ["cpu_baseline", "cpu_umap"])
def test_cpu_baselines_report_their_fields(which):
    a = _args()
    batches = B.make_batches(a, 0, 2)
    r = getattr(B, which)(a, batches)
    assert r["value"] > 0 and r["unit"] == "Mops/s" and r["cores"] >= 1
    assert r["kind"] in ("port", "std::unordered_map replay") and r["sample"]
    if which == "cpu_umap":
        assert r["sharded_value"] > 0 and r["sharded_cores"] >= 1
