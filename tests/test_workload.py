"""CPU checks of the seeded workload generators."""
from __future__ import annotations

import numpy as np

from lslab_b200 import workload as W


def test_splitmix64_known_vector():
    # SplitMix64 seeded with 0: first outputs of the published generator
    got = W.splitmix64(0, 0, 3)
    assert [hex(int(x)) for x in got] == ["0xe220a8397b1dcdaf", "0x6e789e6aa1b965f4",
                                          "0x6c45d188009454f"]


def test_counter_form_is_random_access():
    a = W.splitmix64(7, 0, 100)
    b = W.splitmix64(7, 40, 10)
    assert np.array_equal(a[40:50], b)
    assert np.array_equal(W.key_of_rank(3, np.arange(20)), W.prefill_keys(3, 20))


def test_zipf_ranks_shape():
    n = 1 << 20
    r = W.zipf_ranks(1 << 26, 0.99, 5, 0, n)
    assert r.min() >= 0 and r.max() < (1 << 26)
    c = np.bincount(r[r < 2], minlength=2) / n
    h = W.zeta(1 << 26, 0.99)
    # ranks 0 and 1 are drawn exactly with probability 1 / ((k+1)^theta * zeta);
    # Gray et al.'s method approximates the rest by a continuous inverse
    want = 1.0 / (np.arange(1, 3) ** 0.99 * h)
    assert np.allclose(c, want, rtol=0.05)
    top = np.mean(r < 1000)
    want_top = np.sum(1.0 / (np.arange(1, 1001) ** 0.99)) / h
    assert abs(top - want_top) < 0.05


def test_zeta_tail_approximation():
    exact = float(np.sum(np.arange(1, (1 << 21) + 1, dtype=np.float64) ** -0.99))
    assert abs(W.zeta(1 << 21, 0.99) - exact) / exact < 1e-9


def test_batches_deterministic_and_type_sorted():
    a = W.map_zipf_batch(1, 3, 4096, 1 << 16, 0.99, (0.95, 0.05))
    b = W.map_zipf_batch(1, 3, 4096, 1 << 16, 0.99, (0.95, 0.05))
    assert np.array_equal(a.keys, b.keys) and np.array_equal(a.types, b.types)
    assert np.all(np.diff(a.types.astype(int)) >= 0)
    assert 0.03 < np.mean(a.types == 1) < 0.07


def test_absent_keys_disjoint():
    p = W.prefill_keys(2, 10000)
    a = W.absent_keys(2, 10000, p)
    assert not np.isin(a, p).any()


def test_lognormal_sizes():
    s = W.lognormal_sizes(3, 4096, 512, 1.5, 1, 1 << 18)
    assert s.min() >= 1 and s.max() <= (1 << 18)
    assert 350 < np.median(s) < 700
