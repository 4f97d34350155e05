"""lsb_map_size_noalloc: the allocation-free live count, for callers that
must not allocate device memory (recording a stream capture, or running
under a fixed pre-reserved memory budget).  Checked through the C-ABI
against lsb_map_size, the allocating entry point, on two calls in a row.

This file is collected last on purpose: the entry point shares one static
device array across calls, and the test must hold both in a fresh process
and after every other test has used the library."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import lslab_b200 as L
from lslab_b200 import _lib
from lslab_b200 import workload as W
from tests.util import dev

pytestmark = pytest.mark.gpu


def _noalloc_count(m, cuda) -> int:
    out = cuda.full((1,), -1, dtype=cuda.int64, device="cuda")
    stream = cuda.cuda.current_stream().cuda_stream
    rc = _lib.lib().lsb_map_size_noalloc(m.handle, out.data_ptr(), stream)
    assert rc == _lib.LSB_OK, _lib.error_string(rc)
    cuda.cuda.synchronize()
    return int(out.item())


def test_size_noalloc_equals_size_on_two_calls(cuda):
    m = L.Map(10, pool_slabs=4096)
    keys = W.prefill_keys(77, 60_000)  # ~58 keys a bucket: chains of several slabs
    m.put(dev(keys), dev(keys))
    first = _noalloc_count(m, cuda)
    assert first == m.size() == len(keys)
    m.remove(dev(keys[::3]))
    second = _noalloc_count(m, cuda)
    assert second == m.size() == len(keys) - len(keys[::3])
    assert m.status() == 0


def test_size_noalloc_refuses_maps_over_its_limit(cuda):
    small = L.Map(20)  # 2^20 buckets: the largest accepted
    assert _noalloc_count(small, cuda) == 0
    big = L.Map(21)
    out = cuda.zeros(1, dtype=cuda.int64, device="cuda")
    rc = _lib.lib().lsb_map_size_noalloc(big.handle, out.data_ptr(), None)
    assert rc == _lib.LSB_ERR_ARG
