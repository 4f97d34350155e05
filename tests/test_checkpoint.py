"""Checkpoint format on the host (no GPU): the Python writer and reader of
the file that lsb_map_save / lsb_map_load use round-trip, reject corrupt
files, and fix the format's constants."""
from __future__ import annotations

import struct

import numpy as np
import pytest

from lslab_b200 import checkpoint as CK
from lslab_b200 import workload as W


def test_round_trip_map_and_set(tmp_path):
    k = W.prefill_keys(1, 1000)
    v = W.prefill_values(k)
    CK.write(tmp_path / "m.ck", CK.Checkpoint(0, 12, k, v, pool_slabs=77, lock_mode=1))
    c = CK.read(tmp_path / "m.ck")
    o = np.argsort(k)
    assert c.container == 0 and c.log2_buckets == 12 and c.pool_slabs == 77 and c.lock_mode == 1
    assert np.array_equal(c.keys, k[o]) and np.array_equal(c.values, v[o])
    s = W.perm32(np.arange(333))
    CK.write(tmp_path / "s.ck", CK.Checkpoint(1, 9, s, None))
    c = CK.read(tmp_path / "s.ck")
    assert c.container == 1 and np.array_equal(c.keys, np.sort(s)) and c.values is None


def test_empty_checkpoint(tmp_path):
    CK.write(tmp_path / "e.ck", CK.Checkpoint(0, 4, np.zeros(0, np.uint64), np.zeros(0, np.uint64)))
    c = CK.read(tmp_path / "e.ck")
    assert len(c.keys) == 0 and (tmp_path / "e.ck").stat().st_size == 56


@pytest.mark.parametrize("damage", ["magic", "record", "truncate", "extra", "count"])
def test_corrupt_files_are_rejected(tmp_path, damage):
    k = W.prefill_keys(2, 100)
    p = tmp_path / "m.ck"
    CK.write(p, CK.Checkpoint(0, 8, k, k))
    b = bytearray(p.read_bytes())
    if damage == "magic":
        b[0] ^= 1
    elif damage == "record":
        b[56 + 16 * 37 + 9] ^= 0x40
    elif damage == "truncate":
        b = b[:-5]
    elif damage == "extra":
        b += b"\0"
    else:
        struct.pack_into("<Q", b, 40, 99)
    p.write_bytes(bytes(b))
    with pytest.raises(ValueError):
        CK.read(p)


def test_checksum_is_order_sensitive_and_pinned():
    a = np.arange(1, 5, dtype="<u8").tobytes()
    b = np.array([2, 1, 3, 4], dtype="<u8").tobytes()
    assert CK.checksum(a) != CK.checksum(b)
    # pinned: one word w at position 0 sums to mix64(w)
    assert CK.checksum(np.array([1], "<u8").tobytes()) == int(CK.mix64(np.array([1], np.uint64))[0])
    assert CK.checksum(b"") == 0
    # a trailing partial word is zero-padded
    assert CK.checksum(b"\x01") == CK.checksum(np.array([1], "<u8").tobytes())
