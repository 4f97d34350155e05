"""ctypes binding of liblsb.so (the C-ABI declared in include/lsb.h).

Loading fails loudly: there is no CPU fallback anywhere in the package.
"""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

from .build import LIB, ROOT

HEADER = ROOT / "include" / "lsb.h"

LSB_OK = 0
LSB_ERR_ARG = 1
LSB_ERR_OOM = 2
LSB_ERR_TIMEOUT = 3
LSB_ERR_CUDA = 4
LSB_ERR_STATE = 5
LSB_ERR_IO = 6

STATUS_OOM = 0x1
STATUS_TIMEOUT = 0x2
STATUS_CHAIN = 0x4
STATUS_BARRIER = 0x8
STATUS_SCRATCH = 0x10

OP_GET = 0
OP_PUT = 1
OP_REMOVE = 2
OP_UPDATE = 3
OP_CONTAINS = 0
OP_INSERT = 1

LOCK_WRITER = 0
LOCK_FREE = 1
LOCK_RW = 2


class LsbError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        super().__init__(f"{what}: {error_string(code)} (code {code})")


class Options(C.Structure):
    _fields_ = [
        ("pool_slabs", C.c_uint64),
        ("max_window", C.c_uint32),
        ("lock_mode", C.c_uint32),
        ("device", C.c_int),
    ]


class Tuning(C.Structure):
    _fields_ = [
        ("block_threads", C.c_uint32),
        ("chunk", C.c_uint32),
        ("prefetch", C.c_uint32),
        ("dedup", C.c_uint32),
        ("fused_split", C.c_uint32),
        ("region_order", C.c_uint32),
        ("warp_probe", C.c_uint32),
        ("overlap", C.c_uint32),
        ("read_order", C.c_uint32),
    ]


class TableView(C.Structure):
    """lsb_table_view: the device-side handles of a table (include/lsb.h)."""
    _fields_ = [
        ("slabs", C.c_void_p),
        ("locks", C.c_void_p),
        ("status", C.c_void_p),
        ("pool", C.c_void_p),
        ("free_stack", C.c_void_p),
        ("mask", C.c_uint32),
        ("lock_mode", C.c_uint32),
        ("chunk", C.c_uint32),
        ("pad", C.c_uint32),
    ]


class ServeOptions(C.Structure):
    _fields_ = [
        ("max_wave_ops", C.c_uint32),
        ("ring_requests", C.c_uint32),
        ("arena_ops", C.c_uint64),
        ("idle_ms", C.c_uint32),
        ("pad", C.c_uint32),
    ]


class ServeStats(C.Structure):
    _fields_ = [
        ("waves", C.c_uint64),
        ("ops", C.c_uint64),
        ("requests", C.c_uint64),
        ("state", C.c_uint32),
        ("pad", C.c_uint32),
        ("gather_ns", C.c_uint64),
        ("engine_ns", C.c_uint64),
        ("tail_ns", C.c_uint64),
        ("wait_ns", C.c_uint64),
    ]


class ServeLoad(C.Structure):
    _fields_ = [
        ("nreq", C.c_uint64),
        ("arrival_ns", C.c_void_p),
        ("pool_index", C.c_void_p),
        ("pool_size", C.c_uint32),
        ("pad", C.c_uint32),
        ("pool_off", C.c_void_p),
        ("pool_n", C.c_void_p),
        ("types", C.c_void_p),
        ("keys", C.c_void_p),
        ("vals", C.c_void_p),
        ("results", C.c_void_p),
    ]


_lib: C.CDLL | None = None

_P = C.c_void_p
_SZ = C.c_size_t
_U64 = C.c_uint64
_U32 = C.c_uint32

# name -> (restype, argtypes)
_SIGS = {
    "lsb_map_create": (C.c_int, [C.c_uint, _U64, C.POINTER(_P)]),
    "lsb_map_create_ex": (C.c_int, [C.c_uint, C.POINTER(Options), C.POINTER(_P)]),
    "lsb_map_destroy": (C.c_int, [_P]),
    "lsb_map_get": (C.c_int, [_P, _P, _P, _SZ, _P]),
    "lsb_map_put": (C.c_int, [_P, _P, _P, _P, _SZ, _P]),
    "lsb_map_put_pairs": (C.c_int, [_P, _P, _P, _SZ, _P]),
    "lsb_map_remove": (C.c_int, [_P, _P, _P, _SZ, _P]),
    "lsb_map_update": (C.c_int, [_P, _P, _P, _SZ, _P]),
    "lsb_kvs_create": (C.c_int, [C.c_uint, C.c_uint64, _P, _P]),
    "lsb_kvs_destroy": (C.c_int, [_P]),
    "lsb_kvs_map": (_P, [_P]),
    "lsb_kvs_put": (C.c_int, [_P, _P, _P, _P, _SZ, _P]),
    "lsb_kvs_get": (C.c_int, [_P, _P, _P, _P, _P, _P, C.c_uint64, _SZ, _P, _P]),
    "lsb_kvs_remove": (C.c_int, [_P, _P, _P, _SZ, _P]),
    "lsb_kvs_usage": (C.c_int, [_P, _P, _P, _P, _P]),
    "lsb_kvs_compact": (C.c_int, [_P, _P]),
    "lsb_map_device_view": (C.c_int, [_P, _P]),
    "lsb_set_device_view": (C.c_int, [_P, _P]),
    "lsb_probe_calibrate": (C.c_int, [_P, _U64, C.c_uint32, _P, _P, _SZ, _U64, _P]),
    "lsb_map_get_v32": (C.c_int, [_P, _P, _P, _SZ, _P]),
    "lsb_map_put_v32": (C.c_int, [_P, _P, _P, _P, _SZ, _P]),
    "lsb_map_put_pairs_v32": (C.c_int, [_P, _P, _P, _SZ, _P]),
    "lsb_map_update_v32": (C.c_int, [_P, _P, _P, _SZ, _P]),
    "lsb_map_compact": (C.c_int, [_P, _P, _P]),
    "lsb_set_compact": (C.c_int, [_P, _P, _P]),
    "lsb_map_save": (C.c_int, [_P, C.c_char_p, _P]),
    "lsb_map_load": (C.c_int, [C.c_char_p, _P, _P, _P]),
    "lsb_set_save": (C.c_int, [_P, C.c_char_p, _P]),
    "lsb_set_load": (C.c_int, [C.c_char_p, _P, _P, _P]),
    "lsb_map_execute": (C.c_int, [_P, _P, _P, _P, _P, _SZ, _P]),
    "lsb_map_execute_fused": (C.c_int, [_P, _P, _P, _P, _P, _SZ, _P]),
    "lsb_map_buckets": (_U32, [_P]),
    "lsb_map_get_tuning": (C.c_int, [_P, C.POINTER(Tuning)]),
    "lsb_map_set_tuning": (C.c_int, [_P, C.POINTER(Tuning)]),
    "lsb_map_set_trace": (C.c_int, [_P, C.c_int]),
    "lsb_map_read_trace": (C.c_int, [_P, _P, _SZ, C.POINTER(_SZ), _P]),
    "lsb_map_status": (C.c_int, [_P, C.POINTER(_U32), _P]),
    "lsb_map_pool_usage": (C.c_int, [_P, C.POINTER(_U64), C.POINTER(_U64), _P]),
    "lsb_map_size": (C.c_int, [_P, C.POINTER(_U64), _P]),
    "lsb_map_size_noalloc": (C.c_int, [_P, _P, _P]),
    "lsb_map_dump": (C.c_int, [_P, _P, _P, _SZ, C.POINTER(_U64), _P]),
    "lsb_set_create": (C.c_int, [C.c_uint, _U64, C.POINTER(_P)]),
    "lsb_set_create_ex": (C.c_int, [C.c_uint, C.POINTER(Options), C.POINTER(_P)]),
    "lsb_set_destroy": (C.c_int, [_P]),
    "lsb_set_insert": (C.c_int, [_P, _P, _P, _SZ, _P]),
    "lsb_set_contains": (C.c_int, [_P, _P, _P, _SZ, _P]),
    "lsb_set_remove": (C.c_int, [_P, _P, _P, _SZ, _P]),
    "lsb_set_execute": (C.c_int, [_P, _P, _P, _P, _SZ, _P]),
    "lsb_set_execute_fused": (C.c_int, [_P, _P, _P, _P, _SZ, _P]),
    "lsb_set_buckets": (_U32, [_P]),
    "lsb_set_get_tuning": (C.c_int, [_P, C.POINTER(Tuning)]),
    "lsb_set_set_tuning": (C.c_int, [_P, C.POINTER(Tuning)]),
    "lsb_set_set_trace": (C.c_int, [_P, C.c_int]),
    "lsb_set_read_trace": (C.c_int, [_P, _P, _SZ, C.POINTER(_SZ), _P]),
    "lsb_set_status": (C.c_int, [_P, C.POINTER(_U32), _P]),
    "lsb_set_pool_usage": (C.c_int, [_P, C.POINTER(_U64), C.POINTER(_U64), _P]),
    "lsb_set_size": (C.c_int, [_P, C.POINTER(_U64), _P]),
    "lsb_set_dump": (C.c_int, [_P, _P, _SZ, C.POINTER(_U64), _P]),
    "lsb_map_autotune": (C.c_int, [_P, _P, _P, _P, _P, _SZ, _P, C.POINTER(Tuning)]),
    "lsb_set_autotune": (C.c_int, [_P, _P, _P, _P, _SZ, _P, C.POINTER(Tuning)]),
    "lsb_autotune_lookup": (C.c_int, [C.c_int, C.c_uint, C.POINTER(Tuning)]),
    "lsb_map_capture_fused": (C.c_int, [_P, _P, _P, _P, _P, _SZ, C.POINTER(_P)]),
    "lsb_set_capture_fused": (C.c_int, [_P, _P, _P, _P, _SZ, C.POINTER(_P)]),
    "lsb_graph_launch": (C.c_int, [_P, _P]),
    "lsb_graph_destroy": (C.c_int, [_P]),
    "lsb_serve_create": (C.c_int, [_P, C.POINTER(ServeOptions), C.POINTER(_P)]),
    "lsb_serve_start": (C.c_int, [_P]),
    "lsb_serve_submit": (C.c_int, [_P, _P, _P, _P, _U32, C.POINTER(_U64)]),
    "lsb_serve_poll": (C.c_int, [_P, _U64, C.POINTER(C.c_int)]),
    "lsb_serve_take": (C.c_int, [_P, _U64, _P, C.POINTER(C.c_int)]),
    "lsb_serve_stop": (C.c_int, [_P, C.POINTER(ServeStats)]),
    "lsb_serve_query": (C.c_int, [_P, C.POINTER(ServeStats)]),
    "lsb_serve_destroy": (C.c_int, [_P]),
    "lsb_serve_run_load": (C.c_int, [_P, C.POINTER(ServeLoad), _P, C.POINTER(_U64)]),
    "lsb_error_string": (C.c_char_p, [C.c_int]),
    "lsb_version": (C.c_int, []),
}


def header_symbols() -> list[str]:
    """Function names declared in include/lsb.h."""
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lsb_[a-z0-9_]+)\s*\(", text)))


def lib() -> C.CDLL:
    """Load liblsb.so (built in-tree); raises if it is missing."""
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise RuntimeError(
                f"{LIB} is missing: build it with `python -m lslab_b200.build` "
                "(the package has no CPU fallback)")
        h = C.CDLL(str(LIB))
        for name, (res, args) in _SIGS.items():
            f = getattr(h, name)
            f.restype = res
            f.argtypes = args
        _lib = h
    return _lib


def error_string(code: int) -> str:
    try:
        return lib().lsb_error_string(code).decode()
    except Exception:  # the library itself failed to load
        return f"error {code}"


def check(code: int, what: str) -> None:
    if code != LSB_OK:
        raise LsbError(code, what)
