"""lslab_b200 — B200-native slab-list hash map and set.

Python mirror of the reference's host API (depaulmillz/lslab):

    lslab::map<K,V>::map(n_log_2[, Allocator(pool)])   -> Map(n_log_2, pool_slabs)
    map.put<bs>(keys, values, old_out, size, stream)   -> Map.put(...)
    map.put<bs>(pairs, old_out, size, stream)          -> Map.put_pairs(...)
    map.get<bs>(keys, pair<bool,V>* out, size, stream) -> Map.get(...)
    map.update<bs>(pairs, pair<bool,V>* out, size, s)  -> Map.update(...) (update-if-present)
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
                   OP_REMOVE, OP_UPDATE, STATUS_BARRIER, STATUS_CHAIN, STATUS_OOM, STATUS_SCRATCH, STATUS_TIMEOUT,
                   LsbError)

__all__ = [
    "Map", "Set", "Server", "KVStore", "LsbError", "OP_GET", "OP_PUT", "OP_REMOVE", "OP_UPDATE", "OP_CONTAINS",
    "OP_INSERT",
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

    def device_view(self) -> dict:
        """The table's device handles (lsb_*_device_view): slab array pointer,
        bucket mask, lock mode, ... as a dict of ints."""
        v = _lib.TableView()
        self._call("device_view", C.byref(v))
        return {f: int(getattr(v, f) or 0) for f, _ in _lib.TableView._fields_}

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

    def compact(self, stream=None) -> int:
        """Pack every chain and return emptied overflow slabs to the pool;
        returns the slabs freed (synchronises)."""
        v = C.c_uint64()
        self._call("compact", C.byref(v), _stream(stream))
        return int(v.value)

    def save(self, path, stream=None) -> None:
        """Write the live entries to a checkpoint file (synchronises)."""
        self._call("save", str(path).encode(), _stream(stream))

    @classmethod
    def load(cls, path, pool_slabs: int = 0, *, max_window: int = 0, lock_mode=None,
             device: int = -1, stream=None):
        """A new table holding a checkpoint's entries: the saved shape, or
        the given options (pool_slabs 0 = the saved pool size)."""
        self = cls.__new__(cls)
        self._h = None
        h = C.c_void_p()
        opts = None
        if lock_mode is not None or max_window or pool_slabs or device >= 0:
            opts = C.byref(_opts(pool_slabs, max_window, lock_mode or "writer", device))
        _lib.check(getattr(lib(), f"lsb_{cls._prefix}_load")(str(path).encode(), opts,
                                                              C.byref(h), _stream(stream)),
                   f"lsb_{cls._prefix}_load")
        self._h = h
        self.n_log_2 = (self.buckets() - 1).bit_length()
        return self

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


def probe_calibrate(slabs: int, nslabs: int, slab_bytes: int, req, out, seed: int = 0,
                    size=None, stream=None) -> None:
    """lsb_probe_calibrate: the accesses of one get at a uniformly random key
    per element of `req` over a slab array (see include/lsb.h)."""
    _lib.check(lib().lsb_probe_calibrate(int(slabs), int(nslabs), int(slab_bytes), _ptr(req),
                                         _ptr(out), _len(req, size), int(seed) & (2**64 - 1),
                                         _stream(stream)), "lsb_probe_calibrate")


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

    def update(self, pairs, output=None, size=None, stream=None):
        """Update-if-present of (key, value) pairs (int64 tensor of shape
        (n, 2)); output[i] = {present, old value or 0}."""
        n = size if size is not None else (pairs.numel() // 2)
        self._call("update", _ptr(pairs), _ptr(output), int(n), _stream(stream))

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


class Server:
    """Device-resident request loop over a Map (lsb_serve_*, include/lsb.h).

    Requests are host numpy arrays (types uint8, keys/values uint64); results
    come back as numpy structured arrays of lsb_result.  While the loop runs,
    the map must not be used by other calls."""

    RESULT = None

    def __init__(self, m: "Map", max_wave_ops: int = 0, ring_requests: int = 0,
                 arena_ops: int = 0, idle_ms: int = 0):
        import numpy as np
        if Server.RESULT is None:
            Server.RESULT = np.dtype([("found", "u1"), ("pad", "u1", (7,)), ("value", "<u8")])
        o = _lib.ServeOptions(int(max_wave_ops), int(ring_requests), int(arena_ops),
                              int(idle_ms), 0)
        h = C.c_void_p()
        _lib.check(lib().lsb_serve_create(m._h, C.byref(o), C.byref(h)), "lsb_serve_create")
        self._h = h
        self.map = m

    def start(self):
        _lib.check(lib().lsb_serve_start(self._h), "lsb_serve_start")

    def submit(self, types, keys, values=None) -> int | None:
        """Queue one request; returns its ticket, or None when the queue is full."""
        import numpy as np
        k = np.ascontiguousarray(keys, np.uint64)
        t = None if types is None else np.ascontiguousarray(types, np.uint8)
        v = None if values is None else np.ascontiguousarray(values, np.uint64)
        ticket = C.c_uint64()
        rc = lib().lsb_serve_submit(self._h, None if t is None else t.ctypes.data, k.ctypes.data,
                                    None if v is None else v.ctypes.data, len(k),
                                    C.byref(ticket))
        if rc == _lib.LSB_ERR_STATE:
            return None
        _lib.check(rc, "lsb_serve_submit")
        return int(ticket.value)

    def done(self, ticket: int) -> bool:
        d = C.c_int()
        _lib.check(lib().lsb_serve_poll(self._h, int(ticket), C.byref(d)), "lsb_serve_poll")
        return bool(d.value)

    def take(self, ticket: int, n: int):
        """(results, status) of a finished request of n ops."""
        import numpy as np
        out = np.zeros(n, Server.RESULT)
        st = C.c_int()
        _lib.check(lib().lsb_serve_take(self._h, int(ticket), out.ctypes.data, C.byref(st)),
                   "lsb_serve_take")
        return out, int(st.value)

    def run_load(self, arrival_ns, pool_index, pool_off, pool_n, types, keys, values,
                 want_results: bool = False):
        """Open-loop run (lsb_serve_run_load): latencies (ns per request), wall
        time (ns) and, if asked, all results in issue order."""
        import numpy as np
        arr = np.ascontiguousarray(arrival_ns, np.uint64)
        idx = np.ascontiguousarray(pool_index, np.uint32)
        poff = np.ascontiguousarray(pool_off, np.uint64)
        pn = np.ascontiguousarray(pool_n, np.uint32)
        t = np.ascontiguousarray(types, np.uint8)
        k = np.ascontiguousarray(keys, np.uint64)
        v = np.ascontiguousarray(values, np.uint64)
        res = np.zeros(int(pn[idx].sum()), Server.RESULT) if want_results else None
        lat = np.zeros(len(arr), np.uint64)
        ld = _lib.ServeLoad(len(arr), arr.ctypes.data, idx.ctypes.data, len(pn), 0,
                            poff.ctypes.data, pn.ctypes.data, t.ctypes.data, k.ctypes.data,
                            v.ctypes.data, None if res is None else res.ctypes.data)
        wall = C.c_uint64()
        _lib.check(lib().lsb_serve_run_load(self._h, C.byref(ld), lat.ctypes.data, C.byref(wall)),
                   "lsb_serve_run_load")
        return lat, int(wall.value), res

    @staticmethod
    def _stats(s) -> dict:
        return {"waves": s.waves, "ops": s.ops, "requests": s.requests, "state": s.state,
                "gather_ns": s.gather_ns, "engine_ns": s.engine_ns, "tail_ns": s.tail_ns,
                "wait_ns": s.wait_ns}

    def stop(self) -> dict:
        s = _lib.ServeStats()
        _lib.check(lib().lsb_serve_stop(self._h, C.byref(s)), "lsb_serve_stop")
        return self._stats(s)

    def query(self) -> dict:
        """The running loop's counters and step times so far (lsb_serve_query)."""
        s = _lib.ServeStats()
        _lib.check(lib().lsb_serve_query(self._h, C.byref(s)), "lsb_serve_query")
        return self._stats(s)

    def close(self):
        if self._h is not None:
            lib().lsb_serve_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class KVStore:
    """Variable-size byte values keyed by uint64 (lsb_kvs_*, include/lsb.h):
    values in a device heap of heap_bytes, the map holding key -> (offset,
    length).  put/get/remove take device tensors; get_values is a host-side
    convenience returning Python bytes."""

    def __init__(self, n_log_2: int, heap_bytes: int, pool_slabs: int = 0, *,
                 max_window: int = 0, lock_mode="writer", device: int = -1):
        self._h = None
        h = C.c_void_p()
        _lib.check(lib().lsb_kvs_create(int(n_log_2), int(heap_bytes),
                                        C.byref(_opts(pool_slabs, max_window, lock_mode, device)),
                                        C.byref(h)), "lsb_kvs_create")
        self._h = h

    def _call(self, name, *args):
        _lib.check(getattr(lib(), f"lsb_kvs_{name}")(self._h, *args), f"lsb_kvs_{name}")

    def close(self):
        if self._h is not None:
            lib().lsb_kvs_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def put(self, keys, vals, val_off, size=None, stream=None):
        """vals: uint8 device buffer of the packed values; val_off: n + 1
        int64 offsets into it."""
        self._call("put", _ptr(keys), _ptr(vals), _ptr(val_off), _len(keys, size), _stream(stream))

    def get(self, keys, len_out, dst_off_out, dst=None, dst_cap=0, found_out=None, size=None,
            stream=None) -> int:
        """Found flags, lengths and destination offsets (and the bytes, into
        dst); returns the bytes all found values need."""
        total = C.c_uint64()
        self._call("get", _ptr(keys), _ptr(found_out), _ptr(len_out), _ptr(dst_off_out), _ptr(dst),
                   int(dst_cap), _len(keys, size), C.byref(total), _stream(stream))
        return int(total.value)

    def remove(self, keys, found_out=None, size=None, stream=None):
        self._call("remove", _ptr(keys), _ptr(found_out), _len(keys, size), _stream(stream))

    def usage(self, stream=None) -> dict:
        u, d, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        self._call("usage", C.byref(u), C.byref(d), C.byref(c), _stream(stream))
        return {"heap_used": int(u.value), "heap_dead": int(d.value), "heap_cap": int(c.value)}

    def compact(self, stream=None):
        self._call("compact", _stream(stream))

    def size(self, stream=None) -> int:
        v = C.c_uint64()
        _lib.check(lib().lsb_map_size(lib().lsb_kvs_map(self._h), C.byref(v), _stream(stream)),
                   "lsb_map_size")
        return int(v.value)
