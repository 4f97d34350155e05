"""Checkpoint files on the host: read and write the format that
lsb_map_save / lsb_map_load and lsb_set_save / lsb_set_load use (see
lslab_b200/csrc/lsb_checkpoint.cu), without a GPU.  A checkpoint holds a
table's live entries as records sorted by key after a 56-byte header, so it
can be inspected, produced from other data, or compared.

Header (little-endian): magic b"LSBCKPT1", u32 version (1), u32 container
(0 map<u64,u64>, 1 set<u32>), u32 log2 buckets, u32 key bytes, u32 value
bytes, u32 lock mode, u64 pool slabs, u64 record count, u64 checksum.
Records: map {u64 key, u64 value}, set {u32 key}.  Checksum: the records as
little-endian u64 words (the last zero-padded), sum over i of
mix64(word_i + i * 0x9E3779B97F4A7C15) mod 2^64, mix64 = MurmurHash3's
64-bit finaliser."""
from __future__ import annotations

import struct
from dataclasses import dataclass

import numpy as np

MAGIC = b"LSBCKPT1"
VERSION = 1
HEADER = struct.Struct("<8sIIIIIIQQQ")
assert HEADER.size == 56
_GOLD = np.uint64(0x9E3779B97F4A7C15)


def mix64(x: np.ndarray) -> np.ndarray:
    x = np.asarray(x, np.uint64).copy()
    with np.errstate(over="ignore"):
        x ^= x >> np.uint64(33)
        x *= np.uint64(0xFF51AFD7ED558CCD)
        x ^= x >> np.uint64(33)
        x *= np.uint64(0xC4CEB9FE1A85EC53)
        x ^= x >> np.uint64(33)
    return x


def checksum(records: bytes) -> int:
    pad = (-len(records)) % 8
    words = np.frombuffer(records + b"\0" * pad, "<u8")
    with np.errstate(over="ignore"):
        x = words + np.arange(len(words), dtype=np.uint64) * _GOLD
    return int(np.sum(mix64(x), dtype=np.uint64))


@dataclass
class Checkpoint:
    container: int          # 0 map, 1 set
    log2_buckets: int
    keys: np.ndarray        # ascending; uint64 (map) or uint32 (set)
    values: np.ndarray | None
    pool_slabs: int = 0
    lock_mode: int = 0


def _records(c: Checkpoint) -> bytes:
    if c.container == 0:
        r = np.empty((len(c.keys), 2), "<u8")
        r[:, 0] = c.keys
        r[:, 1] = c.values
        return r.tobytes()
    return np.asarray(c.keys, "<u4").tobytes()


def write(path, c: Checkpoint) -> None:
    order = np.argsort(c.keys, kind="stable")
    c = Checkpoint(c.container, c.log2_buckets, np.asarray(c.keys)[order],
                   None if c.values is None else np.asarray(c.values)[order],
                   c.pool_slabs, c.lock_mode)
    rec = _records(c)
    kb, vb = (8, 8) if c.container == 0 else (4, 0)
    with open(path, "wb") as f:
        f.write(HEADER.pack(MAGIC, VERSION, c.container, c.log2_buckets, kb, vb, c.lock_mode,
                            c.pool_slabs, len(c.keys), checksum(rec)))
        f.write(rec)


def read(path) -> Checkpoint:
    """Parse and verify a checkpoint; ValueError when it is not a valid one."""
    with open(path, "rb") as f:
        data = f.read()
    if len(data) < HEADER.size:
        raise ValueError("truncated header")
    magic, ver, cont, log2, kb, vb, lock, pool, count, ck = HEADER.unpack_from(data)
    if magic != MAGIC or ver != VERSION or cont not in (0, 1):
        raise ValueError("not a checkpoint (magic, version or container)")
    if (kb, vb) != ((8, 8) if cont == 0 else (4, 0)):
        raise ValueError("key/value widths do not match the container")
    rec = data[HEADER.size:]
    if len(rec) != count * (kb + vb):
        raise ValueError("record count does not match the file size")
    if checksum(rec) != ck:
        raise ValueError("checksum mismatch")
    if cont == 0:
        r = np.frombuffer(rec, "<u8").reshape(-1, 2)
        return Checkpoint(0, log2, r[:, 0].copy(), r[:, 1].copy(), pool, lock)
    return Checkpoint(1, log2, np.frombuffer(rec, "<u4").copy(), None, pool, lock)
