"""lslab_b200 — B200-native slab-list hash map and set.

Python mirror of the reference's host API (depaulmillz/lslab):

    lslab::map<K,V>::map(n_log_2[, Allocator(pool)])   -> Map(n_log_2, pool_slabs)
    map.put<bs>(keys, values, old_out, size, stream)   -> Map.put(...)
    map.put<bs>(pairs, old_out, size, stream)          -> Map.put_pairs(...)
    map.get<bs>(keys, pair<bool,V>* out, size, stream) -> Map.get(...)
    (REMOVE branch of detail::traverse)                -> Map.remove(...)
    map.buckets()                                      -> Map.buckets()
    lslab::set<K>::set(n_log_2[, Allocator(pool)])      -> Set(n_log_2, pool_slabs)
    set.insert/contains/remove<bs>(keys, out, size, s) -> Set.insert/contains/remove

Arrays are device buffers: torch CUDA tensors or raw device pointers (int).
Calls are asynchronous on `stream` (a torch.cuda.Stream, a raw cudaStream_t
int, or None for torch's current stream).  Every call goes through the
C-ABI of include/lsb.h into liblsb.so; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C

from . import _lib
from ._lib import (LOCK_FREE, LOCK_RW, LOCK_WRITER, OP_CONTAINS, OP_GET, OP_INSERT, OP_PUT,
                   OP_REMOVE, STATUS_BARRIER, STATUS_CHAIN, STATUS_OOM, STATUS_SCRATCH, STATUS_TIMEOUT,
                   LsbError)

__all__ = [
    "Map", "Set", "LsbError", "OP_GET", "OP_PUT", "OP_REMOVE", "OP_CONTAINS", "OP_INSERT",
    "LOCK_WRITER", "LOCK_FREE", "LOCK_RW", "STATUS_OOM", "STATUS_TIMEOUT", "STATUS_CHAIN",
    "STATUS_BARRIER", "STATUS_SCRATCH", "lib",
]

lib = _lib.lib
_LOCKS = {"writer": LOCK_WRITER, "free": LOCK_FREE, "rw": LOCK_RW}


def _ptr(x) -> int | None:
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        if not x.is_cuda:
            raise ValueError("device buffers are required (got a CPU tensor)")
        if not x.is_contiguous():
            raise ValueError("buffers must be contiguous")
        return x.data_ptr()
    raise TypeError(f"expected a CUDA tensor or a device pointer, got {type(x).__name__}")


def _len(x, size):
    if size is not None:
        return int(size)
    if hasattr(x, "numel"):
        return int(x.numel())
    raise ValueError("size is required when passing raw pointers")


def _stream(s) -> int | None:
    if s is None:
        try:
            import torch
            return torch.cuda.current_stream().cuda_stream
        except Exception:
            return None
    if isinstance(s, int):
        return s
    return s.cuda_stream


def _opts(pool_slabs, max_window, lock_mode, device):
    o = _lib.Options()
    o.pool_slabs = int(pool_slabs or 0)
    o.max_window = int(max_window or 0)
    o.lock_mode = _LOCKS[lock_mode] if isinstance(lock_mode, str) else int(lock_mode)
    o.device = int(device)
    return o


class _Table:
    _prefix = ""

    def __init__(self, n_log_2: int = 10, pool_slabs: int = 0, *, max_window: int = 0,
                 lock_mode="writer", device: int = -1):
        self._h = None
        h = C.c_void_p()
        fn = getattr(lib(), f"lsb_{self._prefix}_create_ex")
        _lib.check(fn(int(n_log_2), C.byref(_opts(pool_slabs, max_window, lock_mode, device)),
                      C.byref(h)), f"lsb_{self._prefix}_create")
        self._h = h
        self.n_log_2 = int(n_log_2)

    def _call(self, name, *args):
        _lib.check(getattr(lib(), f"lsb_{self._prefix}_{name}")(self._h, *args),
                   f"lsb_{self._prefix}_{name}")

    def close(self):
        if self._h is not None:
            getattr(lib(), f"lsb_{self._prefix}_destroy")(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> int:
        return self._h.value

    def buckets(self) -> int:
        return int(getattr(lib(), f"lsb_{self._prefix}_buckets")(self._h))

    def status(self, stream=None) -> int:
        """Device status bits since the last call (synchronises), then cleared."""
        v = C.c_uint32()
        self._call("status", C.byref(v), _stream(stream))
        return int(v.value)

    def pool_usage(self, stream=None) -> tuple[int, int]:
        u, c = C.c_uint64(), C.c_uint64()
        self._call("pool_usage", C.byref(u), C.byref(c), _stream(stream))
        return int(u.value), int(c.value)

    def size(self, stream=None) -> int:
        v = C.c_uint64()
        self._call("size", C.byref(v), _stream(stream))
        return int(v.value)

    def set_trace(self, on: bool = True) -> None:
        self._call("set_trace", int(bool(on)))

    def read_trace(self, stream=None) -> list[tuple[int, int, int]]:
        """Phase stamps of the last fused launch: (ns, window, phase)."""
        import numpy as np
        buf = np.zeros(1024, np.uint64)
        n = C.c_size_t()
        self._call("read_trace", buf.ctypes.data, len(buf), C.byref(n), _stream(stream))
        return [(int(x) >> 8, (int(x) >> 2) & 0x3F, int(x) & 3) for x in buf[: n.value]]

    def autotune(self, types, keys, values, output, size=None, stream=None) -> dict:
        """Sweep the fused path's launch shape on a sample batch (see lsb.h);
        returns the chosen tuning."""
        t = _lib.Tuning()
        if self._prefix == "map":
            self._call("autotune", _ptr(types), _ptr(keys), _ptr(values), _ptr(output),
                       _len(keys, size), _stream(stream), C.byref(t))
        else:
            self._call("autotune", _ptr(types), _ptr(keys), _ptr(output), _len(keys, size),
                       _stream(stream), C.byref(t))
        return {f: int(getattr(t, f)) for f, _ in _lib.Tuning._fields_}

    def capture_fused(self, types, keys, values, output, size=None) -> "Graph":
        """CUDA graph of execute_fused on these buffers (replay with .launch())."""
        g = C.c_void_p()
        if self._prefix == "map":
            self._call("capture_fused", _ptr(types), _ptr(keys), _ptr(values), _ptr(output),
                       _len(keys, size), C.byref(g))
        else:
            self._call("capture_fused", _ptr(types), _ptr(keys), _ptr(output), _len(keys, size),
                       C.byref(g))
        return Graph(g)

    def tuning(self) -> dict:
        t = _lib.Tuning()
        self._call("get_tuning", C.byref(t))
        return {f: int(getattr(t, f)) for f, _ in _lib.Tuning._fields_}

    def set_tuning(self, **kw) -> None:
        cur = self.tuning()
        cur.update(kw)
        t = _lib.Tuning(**cur)
        self._call("set_tuning", C.byref(t))


class Graph:
    """A captured fused launch (lsb_graph)."""

    def __init__(self, handle):
        self._g = handle

    def launch(self, stream=None):
        _lib.check(lib().lsb_graph_launch(self._g, _stream(stream)), "lsb_graph_launch")

    def close(self):
        if self._g is not None and self._g.value:
            lib().lsb_graph_destroy(self._g)
            self._g = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Map(_Table):
    """map<uint64_t, uint64_t> (include/lslab/map.h:24-234)."""

    _prefix = "map"

    def get(self, keys, output, size=None, stream=None):
        self._call("get", _ptr(keys), _ptr(output), _len(keys, size), _stream(stream))

    def put(self, keys, values, output=None, size=None, stream=None):
        self._call("put", _ptr(keys), _ptr(values), _ptr(output), _len(keys, size),
                   _stream(stream))

    def put_pairs(self, pairs, output=None, size=None, stream=None):
        n = size if size is not None else (pairs.numel() // 2)
        self._call("put_pairs", _ptr(pairs), _ptr(output), int(n), _stream(stream))

    def remove(self, keys, output=None, size=None, stream=None):
        self._call("remove", _ptr(keys), _ptr(output), _len(keys, size), _stream(stream))

    def execute(self, types, keys, values, output, size=None, stream=None):
        self._call("execute", _ptr(types), _ptr(keys), _ptr(values), _ptr(output),
                   _len(keys, size), _stream(stream))

    def execute_fused(self, types, keys, values, output, size=None, stream=None):
        self._call("execute_fused", _ptr(types), _ptr(keys), _ptr(values), _ptr(output),
                   _len(keys, size), _stream(stream))

    def dump(self, stream=None):
        """Live (keys, values) as sorted numpy uint64 arrays (synchronises)."""
        import numpy as np
        n = self.size(stream)
        k = np.empty(n, np.uint64)
        v = np.empty(n, np.uint64)
        cnt = C.c_uint64()
        self._call("dump", k.ctypes.data, v.ctypes.data, n, C.byref(cnt), _stream(stream))
        return k[: cnt.value], v[: cnt.value]


class Set(_Table):
    """set<uint32_t> (include/lslab/set.h:21-134)."""

    _prefix = "set"

    def insert(self, keys, output=None, size=None, stream=None):
        self._call("insert", _ptr(keys), _ptr(output), _len(keys, size), _stream(stream))

    def contains(self, keys, output, size=None, stream=None):
        self._call("contains", _ptr(keys), _ptr(output), _len(keys, size), _stream(stream))

    def remove(self, keys, output=None, size=None, stream=None):
        self._call("remove", _ptr(keys), _ptr(output), _len(keys, size), _stream(stream))

    def execute(self, types, keys, output, size=None, stream=None):
        self._call("execute", _ptr(types), _ptr(keys), _ptr(output), _len(keys, size),
                   _stream(stream))

    def execute_fused(self, types, keys, output, size=None, stream=None):
        self._call("execute_fused", _ptr(types), _ptr(keys), _ptr(output), _len(keys, size),
                   _stream(stream))

    def dump(self, stream=None):
        import numpy as np
        n = self.size(stream)
        k = np.empty(n, np.uint32)
        cnt = C.c_uint64()
        self._call("dump", k.ctypes.data, n, C.byref(cnt), _stream(stream))
        return k[: cnt.value]
