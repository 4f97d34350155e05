"""Test infrastructure, not product code.

Python bindings of the checkers:
  * OracleMap / OracleSet — the plain-C restatement of the reference's slab
    list (lsb_oracle.c), run on the host in op-index order;
  * UmapReplay — the op stream replayed on std::unordered_map (umap_replay.cpp),
    the host replay reported as a CPU baseline;
  * RefMap / RefSet — the reference's OWN kernels (lslab::map / lslab::set,
    built for sm_100a from the reference headers into _ref/liblslab_ref.so)
    behind a small C-ABI harness; these need a GPU.

Only tests/, __graft_entry__.smoke() and bench.py's baseline legs use this
package.  The product (lslab_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "liblsb_oracle.so"
UMAP_LIB = HERE / "libumap_replay.so"
REF_LIB = HERE / "_ref" / "liblslab_ref.so"


def reference_include() -> Path | None:
    """Include directory of the reference sources (depaulmillz/lslab), used
    only to build the reference harness: $LSLAB_REFERENCE (the project root)
    when set, else a checkout named `reference` beside this repository; None
    when neither holds include/lslab."""
    env = os.environ.get("LSLAB_REFERENCE")
    root = Path(env) if env else HERE.parent.parent / "reference"
    inc = root / "include"
    return inc if (inc / "lslab").is_dir() else None


class OResult(C.Structure):
    _fields_ = [("found", C.c_uint8), ("pad", C.c_uint8 * 7), ("value", C.c_uint64)]


RESULT_DTYPE = np.dtype([("found", np.uint8), ("pad", np.uint8, 7), ("value", np.uint64)])
assert RESULT_DTYPE.itemsize == 16

_o = None
_r = None


def build(ref: bool | None = None) -> None:
    """Compile the oracle (always) and the reference harness (when the
    reference headers are present)."""
    subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)
    inc = reference_include()
    if ref is None:
        ref = inc is not None
    if ref:
        if inc is None:
            raise RuntimeError("reference sources not found: set LSLAB_REFERENCE to the "
                               "lslab project root")
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF_INCLUDE={inc}"],
                       check=True)


def _olib():
    global _o
    if _o is None:
        if not ORACLE_LIB.exists():
            build(ref=False)
        L = C.CDLL(str(ORACLE_LIB))
        P, SZ, U64 = C.c_void_p, C.c_size_t, C.c_uint64
        sig = {
            "orc_map_create": (P, [C.c_uint, U64]),
            "orc_map_destroy": (None, [P]),
            "orc_map_get": (None, [P, P, P, SZ]),
            "orc_map_put": (None, [P, P, P, P, SZ]),
            "orc_map_remove": (None, [P, P, P, SZ]),
            "orc_map_update": (None, [P, P, P, P, SZ]),
            "orc_map_mixed": (None, [P, P, P, P, P, SZ]),
            "orc_map_mixed_mt": (C.c_int, [P, P, P, P, P, SZ, C.c_int]),
            "orc_map_size": (SZ, [P]),
            "orc_map_dump": (SZ, [P, P, P, SZ]),
            "orc_map_slabs_used": (U64, [P]),
            "orc_map_error": (C.c_int, [P]),
            "orc_set_create": (P, [C.c_uint, U64]),
            "orc_set_destroy": (None, [P]),
            "orc_set_insert": (None, [P, P, P, SZ]),
            "orc_set_contains": (None, [P, P, P, SZ]),
            "orc_set_remove": (None, [P, P, P, SZ]),
            "orc_set_mixed": (None, [P, P, P, P, SZ]),
            "orc_set_mixed_mt": (C.c_int, [P, P, P, P, SZ, C.c_int]),
            "orc_set_size": (SZ, [P]),
            "orc_set_dump": (SZ, [P, P, SZ]),
            "orc_set_slabs_used": (U64, [P]),
            "orc_set_error": (C.c_int, [P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _o = L
    return _o


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


class OracleMap:
    """Host restatement of lslab::map<uint64_t,uint64_t> (see lsb_oracle.c)."""

    def __init__(self, n_log_2: int, pool_capacity: int = 0):
        self.h = _olib().orc_map_create(n_log_2, pool_capacity)
        if not self.h:
            raise MemoryError("oracle map allocation failed")

    def __del__(self):
        if getattr(self, "h", None):
            _olib().orc_map_destroy(self.h)
            self.h = None

    def get(self, keys):
        keys = np.ascontiguousarray(keys, np.uint64)
        out = np.zeros(len(keys), RESULT_DTYPE)
        _olib().orc_map_get(self.h, _p(keys), _p(out), len(keys))
        return out

    def put(self, keys, vals):
        keys = np.ascontiguousarray(keys, np.uint64)
        vals = np.ascontiguousarray(vals, np.uint64)
        old = np.zeros(len(keys), np.uint64)
        _olib().orc_map_put(self.h, _p(keys), _p(vals), _p(old), len(keys))
        return old

    def remove(self, keys):
        keys = np.ascontiguousarray(keys, np.uint64)
        out = np.zeros(len(keys), RESULT_DTYPE)
        _olib().orc_map_remove(self.h, _p(keys), _p(out), len(keys))
        return out

    def update(self, keys, vals):
        keys = np.ascontiguousarray(keys, np.uint64)
        vals = np.ascontiguousarray(vals, np.uint64)
        out = np.zeros(len(keys), RESULT_DTYPE)
        _olib().orc_map_update(self.h, _p(keys), _p(vals), _p(out), len(keys))
        return out

    def mixed(self, types, keys, vals=None, threads: int = 1):
        types = np.ascontiguousarray(types, np.uint8)
        keys = np.ascontiguousarray(keys, np.uint64)
        vals = None if vals is None else np.ascontiguousarray(vals, np.uint64)
        out = np.zeros(len(keys), RESULT_DTYPE)
        if threads > 1:
            r = _olib().orc_map_mixed_mt(self.h, _p(types), _p(keys), _p(vals), _p(out),
                                         len(keys), threads)
            if r < 0:
                raise MemoryError("oracle pool reservation failed")
        else:
            _olib().orc_map_mixed(self.h, _p(types), _p(keys), _p(vals), _p(out), len(keys))
        return out

    def dump(self):
        n = _olib().orc_map_size(self.h)
        k = np.empty(n, np.uint64)
        v = np.empty(n, np.uint64)
        _olib().orc_map_dump(self.h, _p(k), _p(v), n)
        o = np.argsort(k, kind="stable")
        return k[o], v[o]

    def size(self) -> int:
        return int(_olib().orc_map_size(self.h))

    def slabs_used(self) -> int:
        return int(_olib().orc_map_slabs_used(self.h))

    def error(self) -> int:
        return int(_olib().orc_map_error(self.h))


class OracleSet:
    """Host restatement of lslab::set<uint32_t>."""

    def __init__(self, n_log_2: int, pool_capacity: int = 0):
        self.h = _olib().orc_set_create(n_log_2, pool_capacity)
        if not self.h:
            raise MemoryError("oracle set allocation failed")

    def __del__(self):
        if getattr(self, "h", None):
            _olib().orc_set_destroy(self.h)
            self.h = None

    def _run(self, fn, keys):
        keys = np.ascontiguousarray(keys, np.uint32)
        out = np.zeros(len(keys), np.uint8)
        fn(self.h, _p(keys), _p(out), len(keys))
        return out

    def insert(self, keys):
        return self._run(_olib().orc_set_insert, keys)

    def contains(self, keys):
        return self._run(_olib().orc_set_contains, keys)

    def remove(self, keys):
        return self._run(_olib().orc_set_remove, keys)

    def mixed(self, types, keys, threads: int = 1):
        types = np.ascontiguousarray(types, np.uint8)
        keys = np.ascontiguousarray(keys, np.uint32)
        out = np.zeros(len(keys), np.uint8)
        if threads > 1:
            r = _olib().orc_set_mixed_mt(self.h, _p(types), _p(keys), _p(out), len(keys), threads)
            if r < 0:
                raise MemoryError("oracle pool reservation failed")
        else:
            _olib().orc_set_mixed(self.h, _p(types), _p(keys), _p(out), len(keys))
        return out

    def dump(self):
        n = _olib().orc_set_size(self.h)
        k = np.empty(n, np.uint32)
        _olib().orc_set_dump(self.h, _p(k), n)
        return np.sort(k)

    def size(self) -> int:
        return int(_olib().orc_set_size(self.h))


# ------------------------------------------------------------ reference
_u = None


def _ulib():
    global _u
    if _u is None:
        if not UMAP_LIB.exists():
            build(ref=False)
        L = C.CDLL(str(UMAP_LIB))
        P, U32, U64 = C.c_void_p, C.c_uint32, C.c_uint64
        L.umap_create.restype, L.umap_create.argtypes = P, [U32, P, P, U64]
        L.umap_replay.restype, L.umap_replay.argtypes = C.c_double, [P, P, P, P, U64, U32, P]
        L.umap_size.restype, L.umap_size.argtypes = U64, [P]
        L.umap_destroy.restype, L.umap_destroy.argtypes = None, [P]
        _u = L
    return _u


class UmapReplay:
    """std::unordered_map<uint64_t, uint64_t> split into `shards` maps by key
    hash, prefilled with (keys, vals).  replay() runs a batch in op-index
    order with one thread, or one thread per shard, and returns (seconds,
    results) with results in the oracle's result layout."""

    def __init__(self, keys, vals, shards: int = 1):
        keys = np.ascontiguousarray(keys, np.uint64)
        vals = np.ascontiguousarray(vals, np.uint64)
        self.shards = int(shards)
        self._h = _ulib().umap_create(self.shards, keys.ctypes.data, vals.ctypes.data, len(keys))
        if not self._h:
            raise MemoryError("umap_create failed")

    def replay(self, types, keys, vals, threads: int = 1, want_results: bool = True):
        types = np.ascontiguousarray(types, np.uint8)
        keys = np.ascontiguousarray(keys, np.uint64)
        vals = np.ascontiguousarray(vals, np.uint64)
        out = np.zeros(len(keys), RESULT_DTYPE) if want_results else None
        dt = _ulib().umap_replay(self._h, types.ctypes.data, keys.ctypes.data, vals.ctypes.data,
                                 len(keys), int(threads),
                                 out.ctypes.data if out is not None else None)
        if dt < 0:
            raise ValueError("threads must be 1 or the shard count")
        return dt, out

    def size(self) -> int:
        return int(_ulib().umap_size(self._h))

    def close(self):
        if self._h:
            _ulib().umap_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ref_available() -> bool:
    return REF_LIB.exists()


def _rlib():
    global _r
    if _r is None:
        if not REF_LIB.exists():
            raise RuntimeError(f"{REF_LIB} is missing (built by `make -C oracle ref`)")
        L = C.CDLL(str(REF_LIB))
        P, SZ, U64 = C.c_void_p, C.c_size_t, C.c_uint64
        sig = {
            "lref_map_create": (P, [C.c_uint, U64]),
            "lref_map_destroy": (None, [P]),
            "lref_map_put": (C.c_int, [P, P, P, P, SZ, P]),
            "lref_map_get": (C.c_int, [P, P, P, SZ, P]),
            "lref_map_remove": (C.c_int, [P, P, P, SZ, P]),
            "lref_map_pool_used": (U64, [P]),
            "lref_map_pool_capacity": (U64, [P]),
            "lref_map_dump": (SZ, [P, P, P, SZ]),
            "lref_slab_bytes_map": (SZ, []),
            "lref_slab_bytes_set": (SZ, []),
            "lref_set_create": (P, [C.c_uint, U64]),
            "lref_set_destroy": (None, [P]),
            "lref_set_insert": (C.c_int, [P, P, P, SZ, P]),
            "lref_set_contains": (C.c_int, [P, P, P, SZ, P]),
            "lref_set_remove": (C.c_int, [P, P, P, SZ, P]),
            "lref_set_pool_used": (U64, [P]),
            "lref_set_dump": (SZ, [P, P, SZ]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _r = L
    return _r


def ref_map_pool_bound(log2_buckets: int, insert_keys: np.ndarray) -> int:
    """Upper bound on the overflow slabs the reference map can need when every
    key in `insert_keys` (duplicates included) is inserted: with the identity
    hash (include/lslab/hash.h:12-14) each bucket holds at most
    ceil(inserts/31) slabs, one of them the head."""
    mask = np.uint64((1 << log2_buckets) - 1)
    cnt = np.bincount((np.asarray(insert_keys, np.uint64) & mask).astype(np.int64),
                      minlength=1 << log2_buckets)
    return int(np.sum(np.maximum(0, (cnt + 30) // 31 - 1))) + 64


class RefMap:
    """lslab::map<uint64_t,uint64_t> running the reference's own kernels.
    Buffers are torch CUDA tensors."""

    def __init__(self, n_log_2: int, pool_slabs: int):
        self.h = _rlib().lref_map_create(n_log_2, pool_slabs)
        if not self.h:
            raise RuntimeError("reference map creation failed")

    def close(self):
        if getattr(self, "h", None):
            _rlib().lref_map_destroy(self.h)
            self.h = None

    __del__ = close

    def put(self, keys, vals, old, stream=0):
        """`old` receives every op's prior value (the reference's put kernel
        always writes it, so it is required)."""
        if old is None:
            raise ValueError("the reference's put needs an output buffer")
        r = _rlib().lref_map_put(self.h, keys.data_ptr(), vals.data_ptr(), old.data_ptr(),
                                 keys.numel(), stream)
        assert r == 0, r

    def get(self, keys, out, stream=0):
        r = _rlib().lref_map_get(self.h, keys.data_ptr(), out.data_ptr(), keys.numel(), stream)
        assert r == 0, r

    def remove(self, keys, out, stream=0):
        r = _rlib().lref_map_remove(self.h, keys.data_ptr(), out.data_ptr(), keys.numel(), stream)
        assert r == 0, r

    def pool_used(self) -> int:
        return int(_rlib().lref_map_pool_used(self.h))

    def dump(self):
        n = _rlib().lref_map_dump(self.h, None, None, 0)
        if n == C.c_size_t(-1).value:
            raise RuntimeError("reference dump failed")
        k = np.empty(n, np.uint64)
        v = np.empty(n, np.uint64)
        _rlib().lref_map_dump(self.h, _p(k), _p(v), n)
        o = np.argsort(k, kind="stable")
        return k[o], v[o]


class RefSet:
    def __init__(self, n_log_2: int, pool_slabs: int):
        self.h = _rlib().lref_set_create(n_log_2, pool_slabs)
        if not self.h:
            raise RuntimeError("reference set creation failed")

    def close(self):
        if getattr(self, "h", None):
            _rlib().lref_set_destroy(self.h)
            self.h = None

    __del__ = close

    def insert(self, keys, out, stream=0):
        assert _rlib().lref_set_insert(self.h, keys.data_ptr(), out.data_ptr(), keys.numel(),
                                       stream) == 0

    def contains(self, keys, out, stream=0):
        assert _rlib().lref_set_contains(self.h, keys.data_ptr(), out.data_ptr(), keys.numel(),
                                         stream) == 0

    def remove(self, keys, out, stream=0):
        assert _rlib().lref_set_remove(self.h, keys.data_ptr(), out.data_ptr(), keys.numel(),
                                       stream) == 0

    def pool_used(self) -> int:
        return int(_rlib().lref_set_pool_used(self.h))

    def dump(self):
        n = _rlib().lref_set_dump(self.h, None, 0)
        k = np.empty(n, np.uint32)
        _rlib().lref_set_dump(self.h, _p(k), n)
        return np.sort(k)
